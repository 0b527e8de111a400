// trainer_internal.h -- what the batched sweep needs from a trainer (trainer.cu).
#pragma once

#include "common.h"
#include "sweep_body.cuh"

namespace lda {

// A resident trainer's kernel arguments over its whole corpus (all docs, all sampler
// tiles), the arrays a sweep zeroes first, and its shape.
struct TrainerView {
    dev::WtArgs wt;
    dev::StatsArgs st;
    dev::DtArgs dt;       // d_begin = 0, d_end = D
    dev::SampleArgs sm;   // all chunks' tiles; iter is the trainer's current iteration
    int device = 0, K = 0, Vd = 0, warps = 0;
    int64_t N = 0, V = 0, D = 0;
    int* n_k = nullptr;
    int* dwt = nullptr;
    int64_t dwt_count = 0;
    double* tile_ll = nullptr;
    int n_stiles = 0, n_wtiles = 0;
    std::vector<int4> s_tiles, w_tiles;  // host copies (sizes give the schedule)
};

int trainer_view(lda_trainer* t, TrainerView* v);
// Advances the trainer's iteration counter and marks its chunks sampled (with LL or not)
// after sweeps run by someone else on its arrays.
int trainer_note_sweeps(lda_trainer* t, int n, int ll_mode, double ll_sum);

}  // namespace lda
