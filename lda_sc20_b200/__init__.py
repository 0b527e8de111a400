"""lda_sc20_b200 -- B200-native collapsed-Gibbs LDA sweep behind EZLDA's driver surface.

Python mirror of the C ABI (include/lda_b200.h).  The names follow EZLDA's driver
(asherliu/LDA_SC20, EZLDA/mainKernel.cu): a corpus in the word-sorted chunk layout
(EZLDA's Document/DocChunk), a trainer holding the device state (DTChunk, WTAll, WTD)
and the per-stage entry points of one sweep (UpdateWTKernel..., MaxTopicKernel,
UpdateDTKernel, SampleKernel*, PerplexityKernel).  Every call goes to the native
library; nothing here computes on the host.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from ._native import (CorpusInfo, GenConfig, LdaError, SweepCounters, StageTiming, TrainConfig, WordSide,
                      check, load)

__all__ = ["Corpus", "Trainer", "GenConfig", "LdaError", "corpus_config", "load"]

F_TOK_WORD, F_TOK_DOC, F_TOPICS, F_DOC_OFF, F_DTOK_POS, F_DTOK_WORD = 0, 1, 2, 3, 4, 5
F_CHUNK_TOK, F_CHUNK_DOC, F_WORD_COUNT, F_SEG_OFF, F_SEG_CNT = 6, 7, 8, 9, 10


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def corpus_config(name: str, **over) -> GenConfig:
    """Generator presets of the synthetic corpora (seeded stand-ins for EZLDA's PubMed /
    NYTimes runs, whose data are not available).

    c0: D=2,000, V=5,000, len~Poisson(100) in [10,400], 32 generating topics,
        phi~Dir(0.01), theta~Dir(0.1), K=64, dense words: count >= K.
    c1: D=300,000, V=100,000, len~lognormal(5.3,0.6) in [20,2000], 256 generating
        topics, phi~Dir(0.05*V*z) with z a Zipf(1.05) base over word rank, theta~Dir(0.1),
        K=1024, dense words: top 2% by frequency, 8 chunks.
    c2: D=1,000,000, V=1,000,000, len~Poisson(250), 1,000 generating topics with c1's
        phi prior in its urn form, K=10,000, dense words: top 20,000, 8 chunks
        (alpha=0.1 for this corpus).
    """
    presets = {
        "c0": dict(num_docs=2000, vocab=5000, gen_topics=32, len_kind=0, len_p1=100.0, len_p2=0.0,
                   len_min=10, len_max=400, phi_kind=0, phi_conc=0.01, phi_zipf_s=0.0,
                   theta_conc=0.1, K=64, dense_kind=0, dense_param=0.0, num_chunks=1,
                   corpus_seed=1000, topic_seed=42),
        "c1": dict(num_docs=300000, vocab=100000, gen_topics=256, len_kind=1, len_p1=5.3, len_p2=0.6,
                   len_min=20, len_max=2000, phi_kind=1, phi_conc=0.05, phi_zipf_s=1.05,
                   theta_conc=0.1, K=1024, dense_kind=1, dense_param=0.02, num_chunks=8,
                   corpus_seed=1001, topic_seed=42),
    }
    # c1 at one fifth of the documents (~14M tokens): same distributions, sized for
    # profiler captures that must still exceed the 126 MB L2
    presets["c1s"] = dict(presets["c1"], num_docs=60000, vocab=60000)
    # c2: the large-K corpus, D=1,000,000, V=1,000,000, len~Poisson(250) (~250M tokens),
    # 1,000 generating topics with c1's Zipf base in the urn form, K=10,000, the top
    # 20,000 words dense, 8 chunks
    presets["c2"] = dict(num_docs=1000000, vocab=1000000, gen_topics=1000, len_kind=0, len_p1=250.0,
                         len_p2=0.0, len_min=1, len_max=2000, phi_kind=2, phi_conc=0.05, phi_zipf_s=1.05,
                         theta_conc=0.1, K=10000, dense_kind=2, dense_param=20000.0, num_chunks=8,
                         corpus_seed=1002, topic_seed=42)
    # c2 at one tenth of the documents and a fifth of the vocabulary (~25M tokens), for
    # profiler captures of the large-K kernels
    presets["c2s"] = dict(presets["c2"], num_docs=100000, vocab=200000, dense_param=4000.0)
    if name not in presets:
        raise KeyError(f"unknown corpus preset {name!r} (have {sorted(presets)})")
    d = dict(presets[name])
    d.update(over)
    return GenConfig(**d)


class Corpus:
    """Host corpus in EZLDA's word-sorted chunk layout (EZLDA/DataChunk.cuh:22)."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle
        self._lib = load()

    # -- construction
    @classmethod
    def generate(cls, cfg: GenConfig) -> "Corpus":
        h = C.c_void_p()
        check(load().lda_corpus_generate(C.byref(cfg), C.byref(h)))
        return cls(h)

    @classmethod
    def load_ezlda(cls, path: str) -> "Corpus":
        """Reads an EZLDA chunk directory (Document::loadDocument, EZLDA/Doc.cu:45-108)."""
        h = C.c_void_p()
        check(load().lda_corpus_load_ezlda(path.encode(), C.byref(h)))
        return cls(h)

    @classmethod
    def from_docs(cls, doc_off, words, vocab: int, K: int, topics=None, num_chunks: int = 1,
                  dense_kind: int = 0, dense_param: float = 0.0, topic_seed: int = 42) -> "Corpus":
        doc_off = np.ascontiguousarray(doc_off, dtype=np.int64)
        words = np.ascontiguousarray(words, dtype=np.int32)
        tp = None
        if topics is not None:
            topics = np.ascontiguousarray(topics, dtype=np.uint16)
            tp = _ptr(topics)
        h = C.c_void_p()
        check(load().lda_corpus_from_docs(len(doc_off) - 1, _ptr(doc_off), _ptr(words), vocab, tp, K,
                                          num_chunks, dense_kind, dense_param, topic_seed, C.byref(h)))
        return cls(h)

    def write_ezlda(self, path: str, K: int) -> None:
        check(self._lib.lda_corpus_write_ezlda(self._h, path.encode(), K))

    def close(self) -> None:
        if self._h:
            self._lib.lda_corpus_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- inspection
    @property
    def info(self) -> CorpusInfo:
        i = CorpusInfo()
        check(self._lib.lda_corpus_info_get(self._h, C.byref(i)))
        return i

    def _get(self, field: int, dtype, n: int) -> np.ndarray:
        a = np.empty(n, dtype=dtype)
        check(self._lib.lda_corpus_get(self._h, field, _ptr(a), n))
        return a

    @property
    def num_tokens(self) -> int:
        return self.info.num_tokens

    def tok_word(self): return self._get(F_TOK_WORD, np.int32, self.info.num_tokens)
    def tok_doc(self): return self._get(F_TOK_DOC, np.int32, self.info.num_tokens)
    def topics(self): return self._get(F_TOPICS, np.uint16, self.info.num_tokens)
    def doc_off(self): return self._get(F_DOC_OFF, np.int64, self.info.num_docs + 1)
    def dtok_pos(self): return self._get(F_DTOK_POS, np.int64, self.info.num_tokens)
    def dtok_word(self): return self._get(F_DTOK_WORD, np.int32, self.info.num_tokens)
    def chunk_tok(self): return self._get(F_CHUNK_TOK, np.int64, self.info.num_chunks + 1)
    def chunk_doc(self): return self._get(F_CHUNK_DOC, np.int64, self.info.num_chunks + 1)
    def word_count(self): return self._get(F_WORD_COUNT, np.int64, self.info.vocab)

    def seg_off(self):
        i = self.info
        return self._get(F_SEG_OFF, np.int64, i.num_chunks * i.vocab).reshape(i.num_chunks, i.vocab)

    def seg_cnt(self):
        i = self.info
        return self._get(F_SEG_CNT, np.int64, i.num_chunks * i.vocab).reshape(i.num_chunks, i.vocab)

    def set_topics(self, z) -> None:
        z = np.ascontiguousarray(z, dtype=np.uint16)
        check(self._lib.lda_corpus_set_topics(self._h, _ptr(z), len(z)))

    def generate_requests(self, n: int, seed: int, len_median: float = 150.0, len_sigma: float = 1.0,
                          len_min: int = 5, len_max: int = 4000) -> tuple[np.ndarray, np.ndarray]:
        """n new documents from this generated corpus' process (its phi, fresh theta),
        lognormal lengths with the given median and sigma clipped to [len_min, len_max]:
        (doc_off[n+1], words) with words as this corpus' frequency ranks."""
        off = np.zeros(n + 1, dtype=np.int64)
        mu = math.log(len_median)
        check(self._lib.lda_corpus_generate_requests(self._h, seed, n, mu, len_sigma, len_min, len_max,
                                                     _ptr(off), None, 0))
        words = np.empty(int(off[-1]), dtype=np.int32)
        check(self._lib.lda_corpus_generate_requests(self._h, seed, n, mu, len_sigma, len_min, len_max,
                                                     _ptr(off), _ptr(words), len(words)))
        return off, words


@dataclass
class SweepStats:
    tokens: int
    early_accept: int
    full: int
    sum_nnz_full: int
    branch_max: int
    branch_s: int
    branch_q: int
    sum_word_nnz: int
    word_tiles_dense: int
    word_tiles_sparse: int
    rows_evaluated: int
    row_entries_read: int


class Trainer:
    """Device-resident collapsed-Gibbs sweep (EZLDA/mainKernel.cu:158-380)."""

    def __init__(self, corpus: Corpus, K: int, alpha: float | None = None, beta: float = 0.01,
                 seed: int = 42, device: int = 0, device_budget: int = 0, stream_mode: int = 0,
                 num_streams: int = 0, num_dense: int = 0):
        self._lib = load()
        if alpha is None:
            alpha = 50.0 / K  # EZLDA/Argument.cuh:9
        cfg = TrainConfig(K=K, alpha=alpha, beta=beta, seed=seed, device=device, device_budget=device_budget,
                          stream_mode=stream_mode, num_streams=num_streams, num_dense=num_dense)
        h = C.c_void_p()
        check(self._lib.lda_trainer_create(corpus._h, C.byref(cfg), C.byref(h)))
        self._h = h
        self.K = K
        self.alpha = float(np.float32(alpha))
        self.beta = float(np.float32(beta))
        info = corpus.info
        self.N, self.V, self.D, self.C, self.Vd = (info.num_tokens, info.vocab, info.num_docs,
                                                   info.num_chunks, info.num_dense)

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.lda_trainer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- driver
    def iterate(self, n: int = 1, ll: bool = False) -> float | None:
        """n sweeps; with ll=True returns the mean per-token log-likelihood of the last sweep."""
        check(self._lib.lda_trainer_iterate(self._h, n, 1 if ll else 0))
        if ll and n > 0:
            s, t = self.loglik()
            return s / t
        return None

    def iterate_host(self, z_in: np.ndarray, z_out: np.ndarray, ll: bool = False) -> float | None:
        out = C.c_double(0.0)
        check(self._lib.lda_iterate_host(self._h, _ptr(z_in), _ptr(z_out), 1 if ll else 0, C.byref(out)))
        return out.value if ll else None

    def iterate_host_async(self, z_in: np.ndarray, z_out: np.ndarray) -> None:
        """One sweep through pinned host buffers without waiting (lda_iterate_host_async).
        Keep both arrays alive and untouched until wait(); pass the previous call's z_out as
        z_in to overlap each chunk's upload with the previous sweep."""
        check(self._lib.lda_iterate_host_async(self._h, _ptr(z_in), _ptr(z_out)))

    def wait(self) -> None:
        """Waits for the sweeps and copies enqueued by iterate_host_async."""
        check(self._lib.lda_trainer_wait(self._h))

    def loglik(self) -> tuple[float, int]:
        s, n = C.c_double(), C.c_int64()
        check(self._lib.lda_trainer_loglik(self._h, C.byref(s), C.byref(n)))
        return s.value, n.value

    @property
    def iteration(self) -> int:
        v = C.c_uint32()
        check(self._lib.lda_trainer_get_iteration(self._h, C.byref(v)))
        return v.value

    @iteration.setter
    def iteration(self, v: int) -> None:
        check(self._lib.lda_trainer_set_iteration(self._h, v))

    def topics(self) -> np.ndarray:
        z = np.empty(self.N, dtype=np.uint16)
        check(self._lib.lda_trainer_get_topics(self._h, _ptr(z), self.N))
        return z

    def set_topics(self, z) -> None:
        z = np.ascontiguousarray(z, dtype=np.uint16)
        check(self._lib.lda_trainer_set_topics(self._h, _ptr(z), len(z)))

    def counters(self) -> SweepStats:
        c = SweepCounters()
        check(self._lib.lda_trainer_counters(self._h, C.byref(c)))
        return SweepStats(c.tokens, c.early_accept, c.full, c.sum_nnz_full, c.branch_max, c.branch_s,
                          c.branch_q, c.sum_word_nnz, c.word_tiles_dense, c.word_tiles_sparse,
                          c.rows_evaluated, c.row_entries_read)

    def set_timing(self, on: bool) -> None:
        check(self._lib.lda_trainer_set_timing(self._h, 1 if on else 0))

    def timing(self) -> StageTiming:
        t = StageTiming()
        check(self._lib.lda_trainer_timing(self._h, C.byref(t)))
        return t

    def reset_stats(self) -> None:
        check(self._lib.lda_trainer_reset_stats(self._h))

    def set_stream(self, stream_ptr: int | None) -> None:
        check(self._lib.lda_trainer_set_stream(self._h, C.c_void_p(stream_ptr or 0)))

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        check(self._lib.lda_trainer_get_stream(self._h, C.byref(s)))
        return s.value or 0

    def set_chunk_range(self, first: int, last: int) -> None:
        """Sample (and rebuild doc rows for) chunks [first, last) only."""
        check(self._lib.lda_trainer_set_chunk_range(self._h, first, last))

    def set_word_range(self, w0: int, w1: int) -> None:
        """Rebuild word-topic rows and word statistics for words [w0, w1) only."""
        check(self._lib.lda_trainer_set_word_range(self._h, w0, w1))

    def word_side(self) -> _native.WordSide:
        """Device addresses of n_k, the word-topic rows and the word statistics."""
        ws = WordSide()
        check(self._lib.lda_trainer_word_side(self._h, C.byref(ws)))
        return ws

    def sweep_chunks(self, ll: bool = False) -> None:
        """One sweep whose word side (update_wt, max_topic) the caller has already made
        current: the chunk range's doc-row rebuilds and sampling, then the LL."""
        check(self._lib.lda_trainer_sweep_chunks(self._h, 1 if ll else 0))

    def topics_device(self) -> tuple[int, int]:
        """(device address, length) of the uint16 topic array."""
        p, n = C.c_void_p(), C.c_int64()
        check(self._lib.lda_trainer_topics_device(self._h, C.byref(p), C.byref(n)))
        return p.value or 0, n.value

    def stream_info(self) -> tuple[bool, int, int]:
        """(streams its chunks, streams, host->device chunk bytes copied so far)."""
        a, b, c = C.c_int32(), C.c_int32(), C.c_int64()
        check(self._lib.lda_trainer_stream_info(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return bool(a.value), b.value, c.value

    @property
    def device_bytes(self) -> int:
        b = C.c_int64()
        check(self._lib.lda_trainer_device_bytes(self._h, C.byref(b)))
        return b.value

    def checkpoint(self, path: str) -> None:
        check(self._lib.lda_trainer_checkpoint(self._h, path.encode()))

    def restore(self, path: str) -> None:
        check(self._lib.lda_trainer_restore(self._h, path.encode()))

    # -- stage entry points (EZLDA's L2 wrappers)
    def update_wt(self) -> None:
        """UpdateWTDenKernel + UpdateWTDenRowSumKernel + UpdateWTKernel + WTAdditionKernel."""
        check(self._lib.lda_update_wt(self._h))

    def max_topic(self) -> None:
        """MaxTopicKernel (EZLDA/SamplingKernel.cu:77-95)."""
        check(self._lib.lda_max_topic(self._h))

    def update_dt(self, chunk: int) -> None:
        """UpdateDTKernel (EZLDA/DTUpdateKernel.cu:3-15)."""
        check(self._lib.lda_update_dt(self._h, chunk))

    def sample_chunk(self, chunk: int, ll: bool = False) -> None:
        """UpdateProbKernelD + SampleKernelD + SampleKernel (EZLDA/SamplingKernel.cu:18-170)."""
        check(self._lib.lda_sample_chunk(self._h, chunk, 1 if ll else 0))

    def perplexity(self) -> float:
        """PerplexityKernel: FP64 LL sum of the chunks sampled with ll=True."""
        out = C.c_double()
        check(self._lib.lda_perplexity(self._h, C.byref(out)))
        return out.value

    def end_sweep(self) -> None:
        check(self._lib.lda_end_sweep(self._h))

    def sync(self) -> None:
        check(self._lib.lda_trainer_sync(self._h))

    # -- device state readback
    def topic_totals(self) -> np.ndarray:
        a = np.empty(self.K, dtype=np.int32)
        check(self._lib.lda_get_topic_totals(self._h, _ptr(a)))
        return a

    def dense_wt(self) -> np.ndarray:
        a = np.empty(max(self.Vd, 0) * self.K, dtype=np.int32)
        check(self._lib.lda_get_dense_wt(self._h, _ptr(a)))
        return a.reshape(self.Vd, self.K)

    def sparse_wt(self) -> tuple[np.ndarray, np.ndarray]:
        off = np.empty(self.V - self.Vd + 1, dtype=np.int64)
        n = check(self._lib.lda_get_sparse_wt(self._h, _ptr(off), None, 0))
        ent = np.empty(max(n, 1), dtype=np.uint32)
        check(self._lib.lda_get_sparse_wt(self._h, _ptr(off), _ptr(ent), len(ent)))
        return off, ent[:n]

    def word_stats(self):
        top2 = np.empty(self.V, dtype=np.uint32)
        k3 = np.empty(self.V, dtype=np.uint32)
        phi4 = np.empty(self.V * 4, dtype=np.float32)
        ql = np.empty(self.V * 32, dtype=np.float32)
        check(self._lib.lda_get_word_stats(self._h, _ptr(top2), _ptr(k3), _ptr(phi4), _ptr(ql)))
        return top2, k3, phi4.reshape(self.V, 4), ql.reshape(self.V, 32)

    def doc_rows(self) -> tuple[np.ndarray, np.ndarray]:
        off = np.empty(self.D + 1, dtype=np.int64)
        n = check(self._lib.lda_get_doc_rows(self._h, _ptr(off), None, 0))
        ent = np.empty(max(n, 1), dtype=np.uint32)
        check(self._lib.lda_get_doc_rows(self._h, _ptr(off), _ptr(ent), len(ent)))
        return off, ent[:n]

    def token_meta(self) -> np.ndarray:
        a = np.empty(self.N, dtype=np.uint32)
        check(self._lib.lda_get_token_meta(self._h, _ptr(a)))
        return a


def mean_loglik(ll_sum: float, n_tokens: int) -> float:
    return ll_sum / n_tokens if n_tokens else math.nan
