"""ctypes binding of the CPU oracle (liblda_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline / reference legs as the checker.  The product package never imports it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liblda_oracle.so")
LANES = 32


class SampleStats(C.Structure):
    _fields_ = [("tokens", C.c_int64), ("early_accept", C.c_int64), ("full", C.c_int64),
                ("sum_nnz_full", C.c_int64), ("branch_max", C.c_int64), ("branch_s", C.c_int64),
                ("branch_q", C.c_int64), ("loglik", C.c_double)]


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} missing: run `python -m lda_sc20_b200.build`")
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.orc_philox4x32_10.argtypes = [P, P, P]
        L.orc_philox4x32_10.restype = None
        L.orc_token_uniform.argtypes = [C.c_uint64, C.c_uint32, C.c_uint64]
        L.orc_token_uniform.restype = C.c_float
        L.orc_init_topic.argtypes = [C.c_uint64, C.c_uint64, C.c_int32]
        L.orc_init_topic.restype = C.c_uint16
        L.orc_create.argtypes = [C.c_int64, C.c_int32, C.c_int32, C.c_int32, P, P, C.c_float, C.c_float, C.c_int32]
        L.orc_create.restype = P
        L.orc_destroy.argtypes = [P]
        L.orc_destroy.restype = None
        L.orc_rebuild.argtypes = [P, P]
        L.orc_get_topic_totals.argtypes = [P, P]
        L.orc_get_word_row.argtypes = [P, C.c_int32, P]
        L.orc_get_word_rows_packed.argtypes = [P, C.c_int32, C.c_int32, P, P, C.c_int64]
        L.orc_get_word_rows_packed.restype = C.c_int64
        L.orc_get_word_stats.argtypes = [P, P, P, P, P]
        L.orc_get_doc_rows.argtypes = [P, P, P, C.c_int64]
        L.orc_get_doc_rows.restype = C.c_int64
        L.orc_get_token_meta.argtypes = [P, P]
        L.orc_get_recip.argtypes = [P, P]
        L.orc_sample.argtypes = [P, P, C.c_uint64, C.c_uint32, C.c_int32, C.c_int32, C.POINTER(SampleStats)]
        L.orc_iterate.argtypes = [P, P, C.c_uint64, C.c_uint32, C.c_int32, C.POINTER(SampleStats)]
        L.orc_token_probs.argtypes = [P, C.c_int64, P]
        L.orc_foldin.argtypes = [P, P, C.c_int32, C.c_uint32, C.c_uint64, C.c_int32, P, P]
        L.orc_foldin_uniform.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32]
        L.orc_foldin_uniform.restype = C.c_float
        L.orc_foldin_init.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_int32]
        L.orc_foldin_init.restype = C.c_uint16
        L.orc_get_phi_row.argtypes = [P, C.c_int32, P]
        L.orc_set_doc_range.argtypes = [P, C.c_int32, C.c_int32]
        L.orc_set_num_dense.argtypes = [P, C.c_int32]
        _lib = L
    return _lib


def _p(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def philox4x32_10(ctr, key):
    c = np.asarray(ctr, dtype=np.uint32)
    k = np.asarray(key, dtype=np.uint32)
    o = np.zeros(4, dtype=np.uint32)
    lib().orc_philox4x32_10(_p(c), _p(k), _p(o))
    return o


class Oracle:
    """Serial/threaded restatement of one EZLDA sweep over a word-sorted corpus."""

    def __init__(self, tok_word, tok_doc, V: int, D: int, K: int, alpha: float, beta: float,
                 nthreads: int = 0, num_dense: int = 0):
        self.tok_word = np.ascontiguousarray(tok_word, dtype=np.int32)
        self.tok_doc = np.ascontiguousarray(tok_doc, dtype=np.int32)
        self.N, self.V, self.D, self.K = len(self.tok_word), V, D, K
        self.alpha = float(np.float32(alpha))
        self.beta = float(np.float32(beta))
        nt = nthreads or (os.cpu_count() or 1)
        self._h = lib().orc_create(self.N, V, D, K, _p(self.tok_word), _p(self.tok_doc),
                                   self.alpha, self.beta, nt)
        if not self._h:
            raise ValueError("orc_create rejected the corpus")
        if lib().orc_set_num_dense(self._h, int(num_dense)):
            raise ValueError(f"bad num_dense {num_dense}")
        self._z = None

    def close(self):
        if self._h:
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def rebuild(self, z: np.ndarray) -> None:
        self._z = np.ascontiguousarray(z, dtype=np.uint16).copy()  # keep alive while the state points at it
        rc = lib().orc_rebuild(self._h, _p(self._z))
        if rc:
            raise ValueError(f"orc_rebuild failed ({rc})")

    def topic_totals(self):
        a = np.empty(self.K, dtype=np.int32)
        lib().orc_get_topic_totals(self._h, _p(a))
        return a

    def recip(self):
        a = np.empty(self.K, dtype=np.float32)
        lib().orc_get_recip(self._h, _p(a))
        return a

    def word_row(self, w: int):
        a = np.empty(self.K, dtype=np.int32)
        lib().orc_get_word_row(self._h, w, _p(a))
        return a

    def word_rows_packed(self, w0: int, w1: int):
        off = np.empty(w1 - w0 + 1, dtype=np.int64)
        cap = self.N + 1
        ent = np.empty(cap, dtype=np.uint32)
        n = lib().orc_get_word_rows_packed(self._h, w0, w1, _p(off), _p(ent), cap)
        if n < 0:
            raise ValueError("word rows")
        return off, ent[:n]

    def word_stats(self):
        top2 = np.empty(self.V, dtype=np.uint32)
        k3 = np.empty(self.V, dtype=np.uint32)
        phi4 = np.empty(self.V * 4, dtype=np.float32)
        ql = np.empty(self.V * LANES, dtype=np.float32)
        lib().orc_get_word_stats(self._h, _p(top2), _p(k3), _p(phi4), _p(ql))
        return top2, k3, phi4.reshape(self.V, 4), ql.reshape(self.V, LANES)

    def doc_rows(self):
        off = np.empty(self.D + 1, dtype=np.int64)
        ent = np.empty(self.N + 1, dtype=np.uint32)
        n = lib().orc_get_doc_rows(self._h, _p(off), _p(ent), self.N + 1)
        if n < 0:
            raise ValueError("doc rows")
        return off, ent[:n]

    def token_meta(self):
        a = np.empty(self.N, dtype=np.uint32)
        lib().orc_get_token_meta(self._h, _p(a))
        return a

    def sample(self, z_out: np.ndarray, seed: int, it: int, ll: bool = False, word_stride: int = 1):
        st = SampleStats()
        rc = lib().orc_sample(self._h, _p(z_out), seed, it, 1 if ll else 0, word_stride, C.byref(st))
        if rc:
            raise ValueError(f"orc_sample failed ({rc})")
        return st

    def iterate(self, z: np.ndarray, seed: int, it: int, ll: bool = False):
        """One sweep in place (rebuild + sample)."""
        assert z.dtype == np.uint16 and z.flags.c_contiguous
        st = SampleStats()
        rc = lib().orc_iterate(self._h, _p(z), seed, it, 1 if ll else 0, C.byref(st))
        if rc:
            raise ValueError(f"orc_iterate failed ({rc})")
        return st

    def set_doc_range(self, d0: int, d1: int) -> None:
        """Sample only the tokens of docs [d0, d1) from now on (the default is all)."""
        if lib().orc_set_doc_range(self._h, d0, d1):
            raise ValueError(f"bad doc range [{d0}, {d1})")

    def token_probs(self, tok: int):
        p = np.empty(self.K, dtype=np.float64)
        lib().orc_token_probs(self._h, tok, _p(p))
        return p

    def foldin(self, words, rid: int, seed: int, sweeps: int):
        """Fold-in of one document against the counts of the last rebuild: (topics, theta)."""
        w = np.ascontiguousarray(words, dtype=np.int32)
        z = np.empty(len(w), dtype=np.uint16)
        th = np.empty(self.K, dtype=np.float32)
        rc = lib().orc_foldin(self._h, _p(w), len(w), rid, seed, sweeps, _p(z), _p(th))
        if rc:
            raise ValueError(f"orc_foldin failed ({rc})")
        return z, th

    def phi_row(self, w: int):
        a = np.empty(self.K, dtype=np.float32)
        lib().orc_get_phi_row(self._h, w, _p(a))
        return a

    @staticmethod
    def token_uniform(seed: int, it: int, tok: int) -> float:
        return lib().orc_token_uniform(seed, it, tok)

    @staticmethod
    def init_topic(seed: int, tok: int, K: int) -> int:
        return lib().orc_init_topic(seed, tok, K)
