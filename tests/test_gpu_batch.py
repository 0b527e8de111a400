"""Batched multi-model sweeps against each model's own trainer, through the C ABI.

Every model's topics after batched sweeps must equal its own trainer's after the same
sweeps, for every tuning; the per-model LL likewise (bit for bit when the sampler work
items are the trainer's tiles); the autotuner must leave topics, iterations and counters
as they were."""
import numpy as np
import pytest

import lda_sc20_b200 as L
from lda_sc20_b200.batch import Batch, batch_corpus_configs

pytestmark = pytest.mark.gpu


def _models(n, seed=3, scale=1.0):
    cfgs = batch_corpus_configs(n, seed=seed)
    out = []
    for g in cfgs:
        g.num_docs = max(20, int(g.num_docs * scale))
        g.vocab = max(200, int(g.vocab * scale))
        out.append((L.Corpus.generate(g), g.K))
    return out


def _trainers(models, **kw):
    return [L.Trainer(c, K=K, seed=11 + i, **kw) for i, (c, K) in enumerate(models)]


@pytest.mark.parametrize("tuning", [(8, 0, 512), (4, 1, 128), (2, 0, 32)])
def test_batch_equals_plain_trainers(tuning):
    models = _models(12, scale=0.3)
    plain = _trainers(models)
    batched = _trainers(models)
    b = Batch(batched, tuning=tuning)
    ll_b = b.iterate(4, ll=True)
    for i, t in enumerate(plain):
        ll_p = t.iterate(4, ll=True)
        assert np.array_equal(t.topics(), batched[i].topics()), f"model {i} (K={models[i][1]})"
        if tuning[2] == 512:
            assert ll_b[i] == ll_p
        else:
            assert abs(ll_b[i] - ll_p) <= 1e-12 * abs(ll_p)
        assert batched[i].iteration == 4
        cp, cb = t.counters(), batched[i].counters()
        assert (cp.tokens, cp.early_accept, cp.branch_q) == (cb.tokens, cb.early_accept, cb.branch_q)
    launches, work = b.stats()
    assert launches == 4 * 7 + 1 and work > 0


def test_autotune_leaves_no_trace_and_dense_split_is_free():
    models = _models(6, seed=5, scale=0.3)
    plain = _trainers(models)
    batched = _trainers(models, num_dense=-1)      # no dense words: results must not change
    b = Batch(batched)
    b.iterate(2)
    best, ms = b.autotune(sweeps_per_trial=1)
    assert best[0] in (4, 8) and best[1] in (0, 1) and best[2] in (128, 256, 512) and ms > 0
    assert b.tuning == best
    assert all(t.iteration == 2 for t in batched)
    b.iterate(3)
    for i, t in enumerate(plain):
        t.iterate(5)
        assert np.array_equal(t.topics(), batched[i].topics()), f"model {i}"
        assert t.counters().tokens == batched[i].counters().tokens


def test_batch_refuses_foreign_sweeps_and_streaming():
    models = _models(3, seed=7, scale=0.2)
    tr = _trainers(models)
    b = Batch(tr)
    b.iterate(1)
    tr[1].iterate(1)
    with pytest.raises(L.LdaError):
        b.iterate(1)
    st = L.Trainer(models[0][0], K=models[0][1], stream_mode=2)
    with pytest.raises(L.LdaError):
        Batch([st])
    with pytest.raises(L.LdaError):
        Batch([tr[0], tr[0]])


def test_dense_rule_tuner_and_rules_change_no_result():
    """The layout tuner picks one of its rules from timings on a sample; a batch built
    under any rule gives the plain trainers' topics."""
    from lda_sc20_b200.batch import dense_words_for, tune_dense_rule
    models = _models(6, seed=9, scale=0.3)
    corpora = [c for c, _ in models]
    Ks = [K for _, K in models]
    seeds = [11 + i for i in range(len(models))]
    rules = (None, -1, 0.5, 4.0)
    best, timings = tune_dense_rule(corpora, Ks, seeds, rules=rules, sample=4, sweeps_per_trial=1)
    assert best in rules and set(timings) == set(rules) and all(v[0] > 0 for v in timings.values())
    plain = _trainers(models)
    for t in plain:
        t.iterate(3)
    for rule in rules:
        trs = [L.Trainer(c, K=K, seed=11 + i, num_dense=dense_words_for(c, K, rule))
               for i, (c, K) in enumerate(models)]
        b = Batch(trs)
        b.iterate(3)
        for i, t in enumerate(plain):
            assert np.array_equal(t.topics(), trs[i].topics()), f"rule {rule}, model {i}"
