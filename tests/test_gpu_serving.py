"""GPU fold-in serving against the CPU oracle, through the C ABI.

The frozen model's phi rows must equal the oracle's word columns bit for bit; every
request's topics after any number of sweeps, and its theta, must equal orc_foldin's; and
a request's result must not depend on the requests it was batched with."""
import numpy as np
import pytest

import lda_sc20_b200 as L
from lda_sc20_b200.serving import Model, Server
from oracle import Oracle

pytestmark = pytest.mark.gpu

SEED = 7


def _trained(K, sweeps=5, preset="c0", **over):
    c = L.Corpus.generate(L.corpus_config(preset, K=K, **over))
    i = c.info
    tr = L.Trainer(c, K=K, seed=42)
    tr.iterate(sweeps)
    o = Oracle(c.tok_word(), c.tok_doc(), i.vocab, i.num_docs, K, tr.alpha, tr.beta, num_dense=i.num_dense)
    o.rebuild(tr.topics())
    return c, tr, o


def _docs(V, lens, seed=3, word_count=None):
    rng = np.random.default_rng(seed)
    out = []
    for n in lens:
        if word_count is not None:
            p = word_count / word_count.sum()
            out.append(rng.choice(V, size=n, p=p).astype(np.int32))
        else:
            out.append(rng.integers(0, V, size=n).astype(np.int32))
    return out


LENS = [1, 2, 31, 32, 33, 64, 100, 257, 1000, 3000]


@pytest.mark.parametrize("K", [16, 64, 1024])
def test_model_phi_matches_oracle(K):
    c, tr, o = _trained(K)
    m = Model(tr)
    assert (m.K, m.V) == (K, c.info.vocab)
    for w in list(range(0, c.info.vocab, max(1, c.info.vocab // 50))) + [c.info.vocab - 1]:
        assert np.array_equal(m.phi(w).view(np.uint32), o.phi_row(w).view(np.uint32)), f"word {w}"


@pytest.mark.parametrize("K,item", [(16, 32), (64, 32), (1024, 32), (64, 256), (1024, 96), (4096, 32)])
def test_foldin_bit_exact(K, item):
    """Work items of `item` tokens: a request spans up to 94 items on different warps.
    K=4096: the trainer's sparse words carry split Q statistics, which the model turns back
    into lane partials from its phi rows (the fold-in's specification)."""
    c, tr, o = _trained(K)
    m = Model(tr)
    sweeps = 12
    docs = _docs(c.info.vocab, LENS, word_count=c.word_count().astype(np.float64))
    s = Server(m, sweeps=sweeps, max_active=64, max_tokens=1 << 16, seed=SEED, item_tokens=item)
    got = s.run(docs)
    for rid, d in enumerate(docs):
        _, th = o.foldin(d, rid, SEED, sweeps)
        assert np.array_equal(got[rid].view(np.uint32), th.view(np.uint32)), f"doc {rid} (len {len(d)})"
        assert abs(float(got[rid].sum()) - 1.0) < 1e-4


def test_foldin_topics_every_sweep():
    c, tr, o = _trained(64)
    m = Model(tr)
    docs = _docs(c.info.vocab, [5, 77, 500], seed=9, word_count=c.word_count().astype(np.float64))
    sweeps = 6
    s = Server(m, sweeps=sweeps, max_active=8, max_tokens=4096, seed=SEED)
    for rid, d in enumerate(docs):
        s.submit(rid, d)
    for step in range(1, sweeps):
        s.step()
        for rid, d in enumerate(docs):
            z, _ = o.foldin(d, rid, SEED, step)
            assert np.array_equal(s.topics(rid, len(d)), z), f"doc {rid} after {step} sweeps"
    s.step()
    done = set()
    while len(done) < len(docs):       # the last step is collected by a later call
        s.step()
        while (r := s.poll()) is not None:
            done.add(r[0])
    assert s.status() == (0, 0, 4096)


def test_alone_equals_mixed():
    """The same request gives identical theta alone (max_active=1) and inside a mixed batch
    that is admitted in another order and over a fragmented token pool."""
    c, tr, o = _trained(1024)
    m = Model(tr)
    sweeps = 10
    docs = _docs(c.info.vocab, [int(x) for x in np.random.default_rng(5).integers(1, 800, size=120)],
                 word_count=c.word_count().astype(np.float64))
    mixed = Server(m, sweeps=sweeps, max_active=40, max_tokens=12000, seed=SEED)
    order = np.random.default_rng(1).permutation(len(docs))
    for rid in order:
        mixed.submit(int(rid), docs[rid])
    res = {}
    while len(res) < len(docs):
        mixed.step()
        while (r := mixed.poll()) is not None:
            res[r[0]] = r[1]
    alone = Server(m, sweeps=sweeps, max_active=1, max_tokens=1000, seed=SEED)
    for rid in (0, 7, 33, 119):
        alone.submit(rid, docs[rid])
        th = None
        while th is None:
            alone.step()
            r = alone.poll()
            if r is not None:
                assert r[0] == rid
                th = r[1]
        assert np.array_equal(th.view(np.uint32), res[rid].view(np.uint32)), f"doc {rid}"


def test_admission_and_errors():
    c, tr, o = _trained(16)
    m = Model(tr)
    s = Server(m, sweeps=3, max_active=2, max_tokens=100, seed=SEED)
    with pytest.raises(L.LdaError):
        s.submit(0, np.array([c.info.vocab], dtype=np.int32))      # word outside the vocabulary
    with pytest.raises(L.LdaError):
        s.submit(0, np.zeros(101, dtype=np.int32))                 # larger than the pool
    with pytest.raises(L.LdaError):
        s.submit(0, np.zeros(0, dtype=np.int32))                   # empty
    for rid in range(4):
        s.submit(rid, np.arange(40, dtype=np.int32) % c.info.vocab)
    s.step()
    q, a, free = s.status()
    assert (q, a, free) == (2, 2, 20)                              # two slots, 80 of 100 tokens
    done = []
    while len(done) < 4:
        s.step()
        while (r := s.poll()) is not None:
            done.append(r[0])
    assert sorted(done) == [0, 1, 2, 3]
    assert s.status() == (0, 0, 100)


def test_generated_requests_fold_in():
    """Held-out documents of the corpus' generative process (lengths up to 4000)."""
    c, tr, o = _trained(64)
    m = Model(tr)
    off, words = c.generate_requests(60, seed=5, len_median=150, len_sigma=1.0, len_min=5, len_max=4000)
    docs = [words[off[i]:off[i + 1]] for i in range(60)]
    s = Server(m, sweeps=5, max_active=16, max_tokens=20000, seed=SEED)
    got = s.run(docs)
    for rid in range(0, 60, 7):
        _, th = o.foldin(docs[rid], rid, SEED, 5)
        assert np.array_equal(got[rid].view(np.uint32), th.view(np.uint32))
    steps, launches = s.stats()
    assert launches == steps > 0


def test_replay_latency_and_results():
    c, tr, o = _trained(1024)
    m = Model(tr)
    sweeps = 8
    lens = np.random.default_rng(2).integers(20, 400, size=200)
    docs = _docs(c.info.vocab, lens, word_count=c.word_count().astype(np.float64))
    off = np.zeros(len(docs) + 1, dtype=np.int64)
    off[1:] = np.cumsum(lens)
    words = np.concatenate(docs)
    arrival = np.sort(np.random.default_rng(4).uniform(0, 0.2, size=len(docs)))
    s = Server(m, sweeps=sweeps, max_active=256, max_tokens=1 << 17, seed=SEED)
    lat, th, wall = s.replay(off, words, arrival, want_theta=True)
    assert np.all(lat > 0) and wall >= arrival[-1]
    for rid in (0, 50, 199):
        _, ref = o.foldin(docs[rid], rid, SEED, sweeps)
        assert np.array_equal(th[rid].view(np.uint32), ref.view(np.uint32))
