"""ctypes binding of liblda_b200.so (the C ABI declared in include/lda_b200.h)."""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liblda_b200.so")


class LdaError(RuntimeError):
    """Raised when a C ABI call returns a negative status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


ERR_NAMES = {
    -1: "LDA_ERR_ARG", -2: "LDA_ERR_IO", -3: "LDA_ERR_FORMAT", -4: "LDA_ERR_NOMEM",
    -5: "LDA_ERR_DEVICE_MEM", -6: "LDA_ERR_CUDA", -7: "LDA_ERR_STATE", -8: "LDA_ERR_DEVICE",
}


class GenConfig(C.Structure):
    _fields_ = [
        ("num_docs", C.c_int64), ("vocab", C.c_int64), ("gen_topics", C.c_int32),
        ("len_kind", C.c_int32), ("len_p1", C.c_double), ("len_p2", C.c_double),
        ("len_min", C.c_int32), ("len_max", C.c_int32),
        ("phi_kind", C.c_int32), ("phi_conc", C.c_double), ("phi_zipf_s", C.c_double),
        ("theta_conc", C.c_double), ("K", C.c_int32),
        ("dense_kind", C.c_int32), ("dense_param", C.c_double), ("num_chunks", C.c_int32),
        ("corpus_seed", C.c_uint64), ("topic_seed", C.c_uint64),
    ]


class CorpusInfo(C.Structure):
    _fields_ = [
        ("num_tokens", C.c_int64), ("vocab", C.c_int64), ("num_docs", C.c_int64),
        ("num_chunks", C.c_int32), ("num_dense", C.c_int32), ("max_doc_len", C.c_int32),
        ("K_hint", C.c_int32),
    ]


class TrainConfig(C.Structure):
    _fields_ = [
        ("K", C.c_int32), ("alpha", C.c_float), ("beta", C.c_float), ("seed", C.c_uint64),
        ("device", C.c_int32), ("device_budget", C.c_int64), ("stream_mode", C.c_int32),
        ("num_streams", C.c_int32), ("num_dense", C.c_int32),
    ]


class BatchTuning(C.Structure):
    _fields_ = [("warps", C.c_int32), ("schedule", C.c_int32), ("tile_tokens", C.c_int32)]


class SweepCounters(C.Structure):
    _fields_ = [(n, C.c_int64) for n in (
        "tokens", "early_accept", "full", "sum_nnz_full", "branch_max", "branch_s", "branch_q",
        "sum_word_nnz", "word_tiles_dense", "word_tiles_sparse", "rows_evaluated", "row_entries_read")]


class StageTiming(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("ms_wt", "ms_stats", "ms_dt", "ms_sample", "ms_ll", "ms_copy")] + \
               [(n, C.c_int64) for n in ("launches_wt", "launches_stats", "launches_dt",
                                         "launches_sample", "launches_ll")]


class SampleIO(C.Structure):
    """lda_sample_io: device buffers of one allocation-free sampling call."""
    _fields_ = [
        ("K", C.c_int32), ("num_dense", C.c_int32), ("vocab", C.c_int32),
        ("alpha", C.c_float), ("beta", C.c_float), ("seed", C.c_uint64), ("iter", C.c_uint32),
        ("ll_mode", C.c_int32), ("num_tiles", C.c_int32),
        ("tiles", C.c_void_p), ("n_k", C.c_void_p), ("dense_wt", C.c_void_p), ("sparse_off", C.c_void_p),
        ("sparse_nnz", C.c_void_p), ("sparse_ent", C.c_void_p), ("top2", C.c_void_p), ("phi4", C.c_void_p),
        ("ql", C.c_void_p), ("tok_doc", C.c_void_p), ("meta", C.c_void_p), ("topics", C.c_void_p),
        ("doc_len", C.c_void_p), ("dt_off", C.c_void_p), ("dt_nnz", C.c_void_p), ("dt_ent", C.c_void_p),
        ("ll_sum", C.c_void_p),
        ("num_tokens", C.c_int64), ("num_docs", C.c_int32), ("num_dt_entries", C.c_int64),
        ("num_sparse_entries", C.c_int64), ("status", C.c_void_p),
    ]


class WordSide(C.Structure):
    """lda_word_side: device addresses of a trainer's word side."""
    _fields_ = [
        ("n_k", C.c_void_p), ("dense_wt", C.c_void_p), ("sparse_ent", C.c_void_p), ("sparse_nnz", C.c_void_p),
        ("sparse_off", C.c_void_p), ("top2", C.c_void_p), ("k3", C.c_void_p), ("phi4", C.c_void_p), ("ql", C.c_void_p),
        ("qtab", C.c_void_p),
        ("K", C.c_int64), ("vocab", C.c_int64), ("num_dense", C.c_int64), ("sparse_capacity", C.c_int64),
        ("qtab_rounds", C.c_int64),
    ]


P = C.c_void_p
I32, I64, U32, U64, F32, F64 = C.c_int32, C.c_int64, C.c_uint32, C.c_uint64, C.c_float, C.c_double

# name: (restype, argtypes)
SIGNATURES = {
    "lda_last_error": (C.c_char_p, []),
    "lda_version": (C.c_char_p, []),
    "lda_corpus_generate": (I32, [C.POINTER(GenConfig), C.POINTER(P)]),
    "lda_corpus_load_ezlda": (I32, [C.c_char_p, C.POINTER(P)]),
    "lda_corpus_write_ezlda": (I32, [P, C.c_char_p, I32]),
    "lda_corpus_from_docs": (I32, [I64, P, P, I64, P, I32, I32, I32, F64, U64, C.POINTER(P)]),
    "lda_corpus_info_get": (I32, [P, C.POINTER(CorpusInfo)]),
    "lda_corpus_get": (I32, [P, I32, P, I64]),
    "lda_corpus_set_topics": (I32, [P, P, I64]),
    "lda_corpus_free": (None, [P]),
    "lda_trainer_create": (I32, [P, C.POINTER(TrainConfig), C.POINTER(P)]),
    "lda_trainer_destroy": (I32, [P]),
    "lda_trainer_set_stream": (I32, [P, P]),
    "lda_trainer_get_stream": (I32, [P, C.POINTER(P)]),
    "lda_trainer_device_bytes": (I32, [P, C.POINTER(I64)]),
    "lda_trainer_set_chunk_range": (I32, [P, I32, I32]),
    "lda_trainer_topics_device": (I32, [P, C.POINTER(P), C.POINTER(I64)]),
    "lda_trainer_set_word_range": (I32, [P, I32, I32]),
    "lda_trainer_word_side": (I32, [P, C.POINTER(WordSide)]),
    "lda_trainer_sweep_chunks": (I32, [P, I32]),
    "lda_trainer_iterate": (I32, [P, I32, I32]),
    "lda_iterate_host": (I32, [P, P, P, I32, C.POINTER(F64)]),
    "lda_iterate_host_async": (I32, [P, P, P]),
    "lda_trainer_wait": (I32, [P]),
    "lda_trainer_loglik": (I32, [P, C.POINTER(F64), C.POINTER(I64)]),
    "lda_trainer_get_topics": (I32, [P, P, I64]),
    "lda_trainer_set_topics": (I32, [P, P, I64]),
    "lda_trainer_get_iteration": (I32, [P, C.POINTER(U32)]),
    "lda_trainer_set_iteration": (I32, [P, U32]),
    "lda_trainer_counters": (I32, [P, C.POINTER(SweepCounters)]),
    "lda_trainer_set_timing": (I32, [P, I32]),
    "lda_trainer_timing": (I32, [P, C.POINTER(StageTiming)]),
    "lda_trainer_reset_stats": (I32, [P]),
    "lda_trainer_checkpoint": (I32, [P, C.c_char_p]),
    "lda_trainer_restore": (I32, [P, C.c_char_p]),
    "lda_update_wt": (I32, [P]),
    "lda_max_topic": (I32, [P]),
    "lda_update_dt": (I32, [P, I32]),
    "lda_sample_chunk": (I32, [P, I32, I32]),
    "lda_perplexity": (I32, [P, C.POINTER(F64)]),
    "lda_end_sweep": (I32, [P]),
    "lda_trainer_sync": (I32, [P]),
    "lda_get_topic_totals": (I32, [P, P]),
    "lda_get_dense_wt": (I32, [P, P]),
    "lda_get_sparse_wt": (I64, [P, P, P, I64]),
    "lda_get_word_stats": (I32, [P, P, P, P, P]),
    "lda_get_doc_rows": (I64, [P, P, P, I64]),
    "lda_get_token_meta": (I32, [P, P]),
    "lda_sample_chunk_noalloc": (I32, [C.POINTER(SampleIO), I32, P]),
    "lda_model_from_trainer": (I32, [P, I64, P]),
    "lda_model_info": (I32, [P, P, P, P]),
    "lda_model_get_phi": (I32, [P, I32, P]),
    "lda_model_free": (None, [P]),
    "lda_server_create": (I32, [P, I64, I32, I32, U64, P]),
    "lda_server_destroy": (I32, [P]),
    "lda_server_submit": (I32, [P, U32, P, I32]),
    "lda_server_step": (I32, [P, P]),
    "lda_server_poll": (I32, [P, P, P, P]),
    "lda_server_status": (I32, [P, P, P, P]),
    "lda_server_get_topics": (I32, [P, U32, P, I32]),
    "lda_trainer_stream_info": (I32, [P, P, P, P]),
    "lda_corpus_generate_requests": (I32, [P, U64, I64, F64, F64, I32, I32, P, P, I64]),
    "lda_batch_create": (I32, [P, I32, P, P]),
    "lda_batch_destroy": (I32, [P]),
    "lda_batch_set_tuning": (I32, [P, P]),
    "lda_batch_get_tuning": (I32, [P, P]),
    "lda_batch_iterate": (I32, [P, I32, I32]),
    "lda_batch_loglik": (I32, [P, P, I32]),
    "lda_batch_stats": (I32, [P, P, P]),
    "lda_batch_autotune": (I32, [P, I32, P, P]),
    "lda_server_set_item_tokens": (I32, [P, I32]),
    "lda_server_stats": (I32, [P, P, P]),
    "lda_serve_replay": (I32, [P, I32, P, P, P, P, P, P]),
}

_lib = None


def load() -> C.CDLL:
    """Loads liblda_b200.so; raises if it has not been built (there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m lda_sc20_b200.build` "
            "(the CUDA path has no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int) -> int:
    if rc < 0:
        msg = load().lda_last_error()
        raise LdaError(int(rc), (msg or b"").decode(errors="replace"))
    return rc
