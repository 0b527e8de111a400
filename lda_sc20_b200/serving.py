"""Fold-in serving: a frozen model of a trainer and a continuous-batching server.

EZLDA trains only; fold-in is its sweep with the word side frozen (p(k) of a token of
word w in a new document ∝ (n_dk + alpha) * phi_wk), run for a fixed number of sweeps
from per-request Philox initial topics.  The server keeps a token pool in HBM and runs
one sweep of every in-flight request per step, admitting new requests as others retire.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._native import check, load


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


class Model:
    """Frozen phi / per-word statistics of a trainer's current topics (device resident)."""

    def __init__(self, trainer, device_budget: int = 0):
        self._lib = load()
        h = C.c_void_p()
        check(self._lib.lda_model_from_trainer(trainer._h, device_budget, C.byref(h)))
        self._h = h
        K, V, b = C.c_int32(), C.c_int64(), C.c_int64()
        check(self._lib.lda_model_info(h, C.byref(K), C.byref(V), C.byref(b)))
        self.K, self.V, self.bytes = K.value, V.value, b.value

    def phi(self, w: int) -> np.ndarray:
        a = np.empty(self.K, dtype=np.float32)
        check(self._lib.lda_model_get_phi(self._h, w, _ptr(a)))
        return a

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.lda_model_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching fold-in over one Model (which must outlive the server)."""

    def __init__(self, model: Model, sweeps: int = 30, max_active: int = 4096, max_tokens: int = 0,
                 seed: int = 7, item_tokens: int = 32):
        self._lib = load()
        self.model = model
        self.K = model.K
        h = C.c_void_p()
        check(self._lib.lda_server_create(model._h, max_tokens, max_active, sweeps, seed, C.byref(h)))
        self._h = h
        if item_tokens != 32:
            check(self._lib.lda_server_set_item_tokens(h, item_tokens))

    def stats(self) -> tuple[int, int]:
        """(steps issued, fold-in kernel launches)."""
        a, b = C.c_int64(), C.c_int64()
        check(self._lib.lda_server_stats(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def submit(self, rid: int, words) -> None:
        w = np.ascontiguousarray(words, dtype=np.int32)
        check(self._lib.lda_server_submit(self._h, rid, _ptr(w), len(w)))

    def step(self) -> int:
        n = C.c_int32()
        check(self._lib.lda_server_step(self._h, C.byref(n)))
        return n.value

    def poll(self):
        """(rid, theta, latency_s) of one finished request, or None."""
        rid, lat = C.c_uint32(), C.c_double()
        th = np.empty(self.K, dtype=np.float32)
        r = check(self._lib.lda_server_poll(self._h, C.byref(rid), _ptr(th), C.byref(lat)))
        return (rid.value, th, lat.value) if r == 1 else None

    def status(self) -> tuple[int, int, int]:
        q, a, f = C.c_int32(), C.c_int32(), C.c_int64()
        check(self._lib.lda_server_status(self._h, C.byref(q), C.byref(a), C.byref(f)))
        return q.value, a.value, f.value

    def topics(self, rid: int, n: int) -> np.ndarray:
        a = np.empty(n, dtype=np.uint16)
        check(self._lib.lda_server_get_topics(self._h, rid, _ptr(a), n))
        return a

    def run(self, docs) -> dict[int, np.ndarray]:
        """Submits docs (list of word arrays, request ids 0..n-1) at once and steps until
        all finish; returns {rid: theta}."""
        for i, d in enumerate(docs):
            self.submit(i, d)
        out: dict[int, np.ndarray] = {}
        while len(out) < len(docs):
            self.step()
            while (r := self.poll()) is not None:
                out[r[0]] = r[1]
        return out

    def replay(self, doc_off, words, arrival_s, want_theta: bool = False):
        """Real-time replay of an arrival schedule; returns (latency_s, theta|None, wall_s)."""
        off = np.ascontiguousarray(doc_off, dtype=np.int64)
        w = np.ascontiguousarray(words, dtype=np.int32)
        arr = np.ascontiguousarray(arrival_s, dtype=np.float64)
        n = len(off) - 1
        lat = np.zeros(n, dtype=np.float64)
        th = np.zeros((n, self.K), dtype=np.float32) if want_theta else None
        wall = C.c_double()
        check(self._lib.lda_serve_replay(self._h, n, _ptr(off), _ptr(w), _ptr(arr), _ptr(lat),
                                         _ptr(th) if th is not None else None, C.byref(wall)))
        return lat, th, wall.value

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.lda_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
