// ezlda_compat -- command-line driver with EZLDA's surface (EZLDA/mainKernel.cu:30-388).
//
//   ezlda_compat <chunk_dir> [--K 1024] [--alpha 50/K] [--beta 0.01] [--iters 100]
//                [--seed 42] [--device 0] [--ll-every 1] [--record FILE]
//                [--checkpoint FILE] [--resume FILE] [--budget-gb G] [--streams S]
//
// Reads the EZLDA chunk directory (lengthVec.txt, docLength.txt, TLLength.txt, TLSplit.txt,
// chunk<c>/...), runs the sweeps on one GPU through the C ABI and prints per sweep
//   iter <i> loglik <mean per-token LL> ms <sweep time> tokens_per_s <N/time>
//   Average Perplexity:<mean per-token LL>
// The second line keeps the format EZLDA prints from LDATrainPerplexityReduce
// (EZLDA/utility.cu:2143); the value is the FP64 log-likelihood of profilePerp
// (profilePerp/utility.cu:2398,2810) instead of EZLDA's token counter.  Per-sweep
// times go to the record file like EZLDA's SamplingDRecord.txt (mainKernel.cu:376).
// Like EZLDA, chunks stream through the device when the corpus exceeds --budget-gb (or
// always with --streams S > 0, on S CUDA streams); otherwise the corpus stays resident.
// Unlike EZLDA (exit() on any error), errors print the library's message and return 1.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "lda_b200.h"

static int die(const char* what) {
    std::fprintf(stderr, "ezlda_compat: %s: %s\n", what, lda_last_error());
    return 1;
}

int main(int argc, char** argv) {
    if (argc < 2 || std::strcmp(argv[1], "--help") == 0) {
        std::fprintf(stderr, "usage: %s <chunk_dir> [--K n] [--alpha a] [--beta b] [--iters n] [--seed s] "
                             "[--device d] [--ll-every n] [--record file] [--checkpoint file] [--resume file] "
                             "[--budget-gb g] [--streams s]\n", argv[0]);
        return 2;
    }
    const char* dir = argv[1];
    int K = 1024, iters = 100, device = 0, ll_every = 1, streams = 0;
    double alpha = -1.0, beta = 0.01, budget_gb = 0.0;
    unsigned long long seed = 42;
    std::string record = "SamplingDRecord.txt", ckpt, resume;
    for (int i = 2; i < argc; ++i) {
        std::string a = argv[i];
        auto next = [&](void) -> const char* {
            if (i + 1 >= argc) { std::fprintf(stderr, "missing value for %s\n", a.c_str()); std::exit(2); }
            return argv[++i];
        };
        if (a == "--K") K = std::atoi(next());
        else if (a == "--alpha") alpha = std::atof(next());
        else if (a == "--beta") beta = std::atof(next());
        else if (a == "--iters") iters = std::atoi(next());
        else if (a == "--seed") seed = std::strtoull(next(), nullptr, 10);
        else if (a == "--device") device = std::atoi(next());
        else if (a == "--ll-every") ll_every = std::atoi(next());
        else if (a == "--record") record = next();
        else if (a == "--checkpoint") ckpt = next();
        else if (a == "--resume") resume = next();
        else if (a == "--budget-gb") budget_gb = std::atof(next());
        else if (a == "--streams") streams = std::atoi(next());
        else { std::fprintf(stderr, "unknown option %s\n", a.c_str()); return 2; }
    }
    if (alpha <= 0) alpha = 50.0 / K;  // EZLDA/Argument.cuh:9
    lda_corpus* corpus = nullptr;
    if (lda_corpus_load_ezlda(dir, &corpus) != LDA_OK) return die("loading the chunk directory");
    lda_corpus_info info;
    lda_corpus_info_get(corpus, &info);
    std::printf("total num of tokens:%lld docs:%lld words:%lld dense words:%d chunks:%d\n", (long long)info.num_tokens,
                (long long)info.num_docs, (long long)info.vocab, info.num_dense, info.num_chunks);
    lda_train_config cfg{};
    cfg.K = K;
    cfg.alpha = (float)alpha;
    cfg.beta = (float)beta;
    cfg.seed = seed;
    cfg.device = device;
    cfg.device_budget = (int64_t)(budget_gb * 1073741824.0);
    cfg.stream_mode = streams > 0 ? 2 : 0;
    cfg.num_streams = streams;
    lda_trainer* tr = nullptr;
    if (lda_trainer_create(corpus, &cfg, &tr) != LDA_OK) return die("creating the trainer");
    lda_corpus_free(corpus);
    if (!resume.empty() && lda_trainer_restore(tr, resume.c_str()) != LDA_OK) return die("restoring");
    int64_t bytes = 0;
    lda_trainer_device_bytes(tr, &bytes);
    std::printf("Total memory usage : %f GB\n", bytes / 1e9);
    int32_t streaming = 0, nstreams = 0;
    lda_trainer_stream_info(tr, &streaming, &nstreams, nullptr);
    if (streaming) std::printf("chunks streamed through %d CUDA streams\n", nstreams);
    FILE* rec = record.empty() ? nullptr : std::fopen(record.c_str(), "w");
    uint32_t it0 = 0;
    lda_trainer_get_iteration(tr, &it0);
    for (int it = 0; it < iters; ++it) {
        const int ll = ll_every > 0 && (it % ll_every == 0 || it == iters - 1);
        lda_trainer_reset_stats(tr);
        auto t0 = std::chrono::steady_clock::now();
        if (lda_trainer_iterate(tr, 1, ll) != LDA_OK) return die("sweep");
        auto t1 = std::chrono::steady_clock::now();
        const double ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
        lda_sweep_counters cnt{};
        lda_trainer_counters(tr, &cnt);
        if (ll) {
            double s = 0;
            int64_t n = 0;
            lda_trainer_loglik(tr, &s, &n);
            std::printf("iter %u loglik %.6f ms %.3f tokens_per_s %.4e early_accept %.4f\n", it0 + it, s / n, ms,
                        info.num_tokens / (ms / 1e3), cnt.tokens ? (double)cnt.early_accept / cnt.tokens : 0.0);
            std::printf("Average Perplexity:%f\n", s / n);
        } else {
            std::printf("iter %u ms %.3f tokens_per_s %.4e early_accept %.4f\n", it0 + it, ms,
                        info.num_tokens / (ms / 1e3), cnt.tokens ? (double)cnt.early_accept / cnt.tokens : 0.0);
        }
        if (rec) std::fprintf(rec, "%f\n", ms);
    }
    if (rec) std::fclose(rec);
    if (!ckpt.empty() && lda_trainer_checkpoint(tr, ckpt.c_str()) != LDA_OK) return die("checkpoint");
    lda_trainer_destroy(tr);
    return 0;
}
