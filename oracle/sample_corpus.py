"""Seeded numpy draw of a synthetic LDA corpus, for the CPU baseline legs of bench.py.

TEST INFRASTRUCTURE ONLY.  The CPU legs time the oracle on the host cores and must not
load the product library, so they cannot use its C++ generator.  This module draws from
the same generative process (the parameters of lda_sc20_b200.corpus_config presets):

  * doc lengths: Poisson(len_p1) (len_kind 0) or round(exp(N(len_p1, len_p2))) (len_kind 1),
    clipped to [len_min, len_max];
  * gen_topics topic-word distributions phi_t ~ Dir(a), a_w = phi_conc (phi_kind 0) or
    phi_conc * V * z_w with z a Zipf(phi_zipf_s) base over word rank (phi_kind 1 and 2);
  * per doc theta_d ~ Dir(theta_conc), each token's topic from theta_d and its word from
    phi of that topic;
  * initial sampler topics uniform over [0, K).

It is the same distribution, not the same corpus: numpy's streams differ from the C++
generator's, so token counts and word ids differ from the product's corpus of the same
preset.  Word ids are relabelled by decreasing frequency, as in the product's layout.
"""
from __future__ import annotations

import numpy as np


def _dirichlet_rows(rng: np.random.Generator, a: np.ndarray, rows: int) -> np.ndarray:
    """rows draws of Dir(a), normalised gamma variates (rows with every variate 0 after
    underflow fall back to the normalised parameter)."""
    g = rng.gamma(np.broadcast_to(a, (rows, len(a))))
    s = g.sum(axis=1, keepdims=True)
    bad = s[:, 0] <= 0
    if bad.any():
        g[bad] = a / a.sum()
        s[bad] = 1.0
    return g / s


def draw_corpus(cfg, num_docs: int, seed: int) -> dict:
    """num_docs documents of the process described by `cfg` (a GenConfig-like object with
    the preset's fields).  Returns tok_word, tok_doc (int32, word-sorted), topics (uint16
    initial topics), and V, D, K."""
    rng = np.random.default_rng(seed)
    V, T, K, D = int(cfg.vocab), int(cfg.gen_topics), int(cfg.K), int(num_docs)
    if cfg.len_kind == 0:
        lens = rng.poisson(cfg.len_p1, size=D)
    else:
        lens = np.rint(np.exp(cfg.len_p1 + cfg.len_p2 * rng.standard_normal(D))).astype(np.int64)
    lens = np.clip(lens, cfg.len_min, cfg.len_max).astype(np.int64)
    N = int(lens.sum())
    if cfg.phi_kind == 0:
        a = np.full(V, float(cfg.phi_conc))
    else:
        z = np.arange(1, V + 1, dtype=np.float64) ** -float(cfg.phi_zipf_s)
        a = float(cfg.phi_conc) * V * z / z.sum()
    doc = np.repeat(np.arange(D, dtype=np.int64), lens)
    # topics: inverse CDF of each doc's theta, searched in the doc-offset cumulative table
    theta = _dirichlet_rows(rng, np.full(T, float(cfg.theta_conc)), D)
    cum = np.cumsum(theta, axis=1)
    cum /= cum[:, -1:]
    flat = (cum + np.arange(D, dtype=np.float64)[:, None]).ravel()
    u = rng.random(N)
    t = np.searchsorted(flat, doc + u, side="right") - doc * T
    t = np.minimum(t, T - 1)
    # words: per generating topic, inverse CDF of its phi
    words = np.empty(N, dtype=np.int64)
    order = np.argsort(t, kind="stable")
    bounds = np.searchsorted(t[order], np.arange(T + 1))
    for k in range(T):
        idx = order[bounds[k]:bounds[k + 1]]
        if len(idx) == 0:
            continue
        phi = _dirichlet_rows(rng, a, 1)[0]
        c = np.cumsum(phi)
        c /= c[-1]
        words[idx] = np.minimum(np.searchsorted(c, rng.random(len(idx)), side="right"), V - 1)
    # relabel words by decreasing frequency (stable), then sort the tokens by (word, doc)
    cnt = np.bincount(words, minlength=V)
    rank_of = np.empty(V, dtype=np.int64)
    rank_of[np.argsort(-cnt, kind="stable")] = np.arange(V)
    words = rank_of[words]
    srt = np.lexsort((doc, words))
    return {"tok_word": words[srt].astype(np.int32), "tok_doc": doc[srt].astype(np.int32),
            "topics": rng.integers(0, K, size=N, dtype=np.uint16), "V": V, "D": D, "K": K, "N": N}
