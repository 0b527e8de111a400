"""Batched training of many independent corpora: one work list per sweep stage spanning
every model, persistent kernels, and the sweeps of a run as one CUDA graph launch.

EZLDA trains one corpus per process; here a batch sweeps resident trainers together.
Each model keeps its own K, alpha, beta and seed, and its topics after a batched sweep
equal its own trainer's after the same sweep.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._native import BatchTuning, check, load


class Batch:
    def __init__(self, trainers, tuning: tuple[int, int, int] | None = None):
        self._lib = load()
        self.trainers = list(trainers)      # the batch needs them alive
        arr = (C.c_void_p * len(self.trainers))(*[t._h.value for t in self.trainers])
        tu = BatchTuning(*tuning) if tuning is not None else None
        h = C.c_void_p()
        check(self._lib.lda_batch_create(arr, len(self.trainers), C.byref(tu) if tu else None, C.byref(h)))
        self._h = h

    @property
    def tuning(self) -> tuple[int, int, int]:
        t = BatchTuning()
        check(self._lib.lda_batch_get_tuning(self._h, C.byref(t)))
        return t.warps, t.schedule, t.tile_tokens

    @tuning.setter
    def tuning(self, v: tuple[int, int, int]) -> None:
        t = BatchTuning(*v)
        check(self._lib.lda_batch_set_tuning(self._h, C.byref(t)))

    def iterate(self, n: int = 1, ll: bool = False):
        """n sweeps of every model in one graph launch; with ll the per-model mean per-token
        log-likelihood of the last sweep."""
        check(self._lib.lda_batch_iterate(self._h, n, 1 if ll else 0))
        if not ll or n == 0:
            return None
        s = self.loglik()
        return s / np.array([t.N for t in self.trainers], dtype=np.float64)

    def loglik(self) -> np.ndarray:
        a = np.empty(len(self.trainers), dtype=np.float64)
        check(self._lib.lda_batch_loglik(self._h, C.c_void_p(a.ctypes.data), len(a)))
        return a

    def stats(self) -> tuple[int, int]:
        """(kernel launches issued, work items per sweep)."""
        a, b = C.c_int64(), C.c_int64()
        check(self._lib.lda_batch_stats(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def autotune(self, sweeps_per_trial: int = 2) -> tuple[tuple[int, int, int], float]:
        t = BatchTuning()
        ms = C.c_double()
        check(self._lib.lda_batch_autotune(self._h, sweeps_per_trial, C.byref(t), C.byref(ms)))
        return (t.warps, t.schedule, t.tile_tokens), ms.value

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.lda_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_corpus_configs(n: int, seed: int = 3):
    """The batched workload's per-model generator configurations: K from
    {16,32,64,128,256}, D ~ U[100,5000], V ~ U[1000,20000], doc lengths Poisson(80),
    16 generating topics with phi ~ Dir(0.01) and theta ~ Dir(0.1), one chunk each."""
    from . import corpus_config
    rng = np.random.default_rng(seed)
    out = []
    for m in range(n):
        K = int(rng.choice([16, 32, 64, 128, 256]))
        D = int(rng.integers(100, 5001))
        V = int(rng.integers(1000, 20001))
        out.append(corpus_config("c0", num_docs=D, vocab=V, gen_topics=16, len_p1=80.0, len_min=1, len_max=400,
                                 K=K, num_chunks=1, corpus_seed=100000 + 7919 * m + seed, topic_seed=42 + m))
    return out


def dense_words_for(corpus, K: int, rule):
    """The trainer's num_dense for a dense-word rule: None keeps the corpus' split, -1 makes
    no word dense, and a float f makes the words with at least f*K tokens dense (words are
    frequency ranks; words above 65535 tokens are dense under every rule)."""
    if rule is None:
        return 0
    wc = corpus.word_count()
    forced = int((wc > 65535).sum())
    if rule == -1:
        return forced if forced else -1
    n = max(int((wc >= rule * K).sum()), forced)
    return n if n else -1


def tune_dense_rule(corpora, Ks, seeds, rules=(None, -1, 0.5, 1.0, 4.0), sample: int = 64,
                    sweeps_per_trial: int = 2, device: int = 0, rng_seed: int = 0):
    """Picks the dense-word rule for a batch: on a random sample of the models, builds a
    batch per rule, lets the batch autotuner pick its best tuning, and keeps the rule
    whose best sweep is fastest.  The rule changes only the layout, never a result.
    Returns (rule, {rule: (ms per sweep, tuning)})."""
    from . import Trainer
    rng = np.random.default_rng(rng_seed)
    idx = rng.choice(len(corpora), size=min(sample, len(corpora)), replace=False)
    timings = {}
    for rule in rules:
        trs = [Trainer(corpora[i], K=Ks[i], seed=seeds[i], device=device,
                       num_dense=dense_words_for(corpora[i], Ks[i], rule)) for i in idx]
        b = Batch(trs)
        tuning, ms = b.autotune(sweeps_per_trial=sweeps_per_trial)
        timings[rule] = (ms, tuning)
        b.close()
        for t in trs:
            t.close()
    best = min(timings, key=lambda r: timings[r][0])
    return best, timings
