"""GPU parity of the CUDA sweep against the CPU oracle, through the C ABI.

Integer state (n_k, dense/sparse word-topic rows, doc rows, per-token metadata) must be
bit-exact; per-word float statistics bit-exact; sampled topics identical token for token
(the kernels and the oracle share one arithmetic specification); the FP64
log-likelihood within 1e-9 relative (summation order differs)."""
import os

import numpy as np
import pytest

import lda_sc20_b200 as L
from oracle import Oracle

pytestmark = pytest.mark.gpu

LL_RTOL = 1e-9


def _setup(corpus, K, seed=42, nthreads=0):
    i = corpus.info
    tr = L.Trainer(corpus, K=K, seed=seed)
    o = Oracle(corpus.tok_word(), corpus.tok_doc(), i.vocab, i.num_docs, K, tr.alpha, tr.beta, nthreads=nthreads,
               num_dense=i.num_dense)
    return tr, o


def _compare_state(tr, o, corpus, check_rows=True):
    i = corpus.info
    assert np.array_equal(tr.topic_totals(), o.topic_totals())
    Vd = i.num_dense
    if Vd:
        dwt = tr.dense_wt()
        for w in range(Vd):
            assert np.array_equal(dwt[w], o.word_row(w)), f"dense word {w}"
    soff, sent = tr.sparse_wt()
    ooff, oent = o.word_rows_packed(Vd, i.vocab)
    assert np.array_equal(soff, ooff)
    assert np.array_equal(sent, oent)
    g = tr.word_stats()
    r = o.word_stats()
    names = ("top2", "k3", "phi4", "ql")
    for a, b, n in zip(g, r, names):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), n
    if check_rows:
        goff, gent = tr.doc_rows()
        roff, rent = o.doc_rows()
        assert np.array_equal(goff, roff)
        assert np.array_equal(gent, rent)
        assert np.array_equal(tr.token_meta(), o.token_meta())


@pytest.mark.parametrize("chunks,dense_kind,dense_param", [(1, 0, 0.0), (3, 1, 0.05)])
def test_stage_parity_one_sweep(chunks, dense_kind, dense_param):
    c = L.Corpus.generate(L.corpus_config("c0", num_chunks=chunks, dense_kind=dense_kind, dense_param=dense_param))
    K = 64
    tr, o = _setup(c, K)
    z0 = c.topics()
    o.rebuild(z0)
    tr.update_wt()
    tr.max_topic()
    for ch in range(c.info.num_chunks):
        tr.update_dt(ch)
    tr.sync()
    _compare_state(tr, o, c)
    for ch in range(c.info.num_chunks):
        tr.sample_chunk(ch, ll=True)
    ll_gpu = tr.perplexity()
    zo = z0.copy()
    st = o.sample(zo, 42, 0, ll=True)
    zg = tr.topics()
    assert np.array_equal(zg, zo), f"{(zg != zo).sum()} of {len(zo)} topics differ"
    assert abs(ll_gpu - st.loglik) <= LL_RTOL * abs(st.loglik)
    cnt = tr.counters()
    assert cnt.tokens == st.tokens and cnt.early_accept == st.early_accept
    assert (cnt.branch_max, cnt.branch_s, cnt.branch_q) == (st.branch_max, st.branch_s, st.branch_q)


def test_fifty_sweeps_bit_exact_c0():
    """Config 0 (K=64, ~200K tokens, 50 sweeps): identical topics after every sweep and
    the LL curve within 1e-9 of the oracle's."""
    c = L.Corpus.generate(L.corpus_config("c0"))
    K = 64
    tr, o = _setup(c, K)
    z = c.topics()
    lls = []
    for it in range(50):
        st = o.iterate(z, 42, it, ll=True)
        ll = tr.iterate(1, ll=True)
        s, n = tr.loglik()
        assert n == len(z)
        assert abs(s - st.loglik) <= LL_RTOL * abs(st.loglik), it
        if it % 5 == 4 or it == 49:
            zg = tr.topics()
            assert np.array_equal(zg, z), f"sweep {it}: {(zg != z).sum()} topics differ"
        lls.append(ll)
    assert lls[-1] > lls[0]  # the chain is mixing toward higher likelihood


@pytest.mark.parametrize("K", [4, 16, 100, 1024, 4096, 10000])
def test_k_variants(K):
    c = L.Corpus.generate(L.corpus_config("c0", num_docs=500, vocab=800, K=K, num_chunks=2))
    tr, o = _setup(c, K)
    z = c.topics()
    tr2 = L.Trainer(c, K=K, seed=7)
    for it in range(3):
        st = o.iterate(z, 7, it, ll=True)
        tr2.iterate(1, ll=True)
        s, _ = tr2.loglik()
        assert abs(s - st.loglik) <= LL_RTOL * abs(st.loglik), f"LL at sweep {it}"
    assert np.array_equal(tr2.topics(), z)
    del tr


@pytest.mark.parametrize("K,preset,alpha,stream_mode", [
    (4096, "c0", None, 1), (4096, "c0", None, 2), (10000, "c1", 0.1, 1), (10000, "c1", 0.1, 2)])
def test_large_k_dense_words_bit_exact(K, preset, alpha, stream_mode):
    """Above 2048 topics dense words go to the CTA-per-tile dense-word sampler and sparse
    words to the column-free one (the path of LDAKernelTrainD + UpdateProbKernelTrainD1,
    EZLDA/utility.cu:1625-2103, :2680-3312, and LDAKernelTrain, :1217-1611).  Corpora with
    dense words, resident and streamed, plain and LL sweeps: topics equal the oracle's token
    for token after every sweep and the FP64 LL is within 1e-9.  The K=10,000 case uses
    Zipfian word frequencies, so frequent dense words span several 2048-token tiles."""
    if preset == "c0":
        cfg = L.corpus_config("c0", num_docs=2000, vocab=5000, K=K, num_chunks=3, dense_kind=1, dense_param=0.05)
    else:
        cfg = L.corpus_config("c1", num_docs=3000, vocab=6000, K=K, num_chunks=3, corpus_seed=99)
    c = L.Corpus.generate(cfg)
    i = c.info
    assert i.num_dense > 0
    tr = L.Trainer(c, K=K, alpha=alpha, seed=11, stream_mode=stream_mode, num_streams=2)
    assert tr.stream_info()[0] is (stream_mode == 2)
    o = Oracle(c.tok_word(), c.tok_doc(), i.vocab, i.num_docs, K, tr.alpha, tr.beta, num_dense=i.num_dense)
    z = c.topics()
    for it in range(3):
        ll = it != 1  # sweeps 0 and 2 run the LL-mode kernels, sweep 1 the plain ones
        st = o.iterate(z, 11, it, ll=ll)
        tr.reset_stats()
        tr.iterate(1, ll=ll)
        if ll:
            s, _ = tr.loglik()
            assert abs(s - st.loglik) <= LL_RTOL * abs(st.loglik), f"LL at sweep {it}"
        zg = tr.topics()
        assert np.array_equal(zg, z), f"sweep {it}: {(zg != z).sum()} of {len(z)} topics differ"
        cnt = tr.counters()
        assert cnt.word_tiles_dense > 0 and cnt.word_tiles_sparse > 0
        assert (cnt.branch_max, cnt.branch_s, cnt.branch_q) == (st.branch_max, st.branch_s, st.branch_q)


def test_mid_size_k1024_lognormal():
    cfg = L.corpus_config("c1", num_docs=20000, vocab=20000, num_chunks=4, corpus_seed=77)
    c = L.Corpus.generate(cfg)
    K = 1024
    tr, o = _setup(c, K)
    z = c.topics()
    for it in range(3):
        st = o.iterate(z, 42, it, ll=True)
        tr.iterate(1, ll=True)
        s, _ = tr.loglik()
        assert abs(s - st.loglik) <= LL_RTOL * abs(st.loglik)
    assert np.array_equal(tr.topics(), z)
    o.rebuild(z)
    tr.update_wt()
    tr.max_topic()
    for ch in range(c.info.num_chunks):
        tr.update_dt(ch)
    tr.sync()
    _compare_state(tr, o, c)


def test_empty_docs_and_tiny_corpus():
    rng = np.random.default_rng(1)
    lens = rng.integers(0, 30, size=64)
    lens[[0, 7, 63]] = 0
    off = np.concatenate([[0], np.cumsum(lens)])
    words = rng.integers(0, 40, size=off[-1]).astype(np.int32)
    c = L.Corpus.from_docs(off, words, vocab=40, K=8, num_chunks=3)
    tr, o = _setup(c, 8)
    z = c.topics()
    for it in range(4):
        o.iterate(z, 42, it)
        tr.iterate(1)
    assert np.array_equal(tr.topics(), z)


def test_host_iterate_matches_resident():
    c = L.Corpus.generate(L.corpus_config("c0"))
    a = L.Trainer(c, K=64)
    b = L.Trainer(c, K=64)
    z = c.topics()
    out = np.empty_like(z)
    for it in range(3):
        lb = b.iterate_host(z, out, ll=True)
        a.iterate(1, ll=True)
        z = out.copy()
        assert abs(a.loglik()[0] - lb) <= 1e-12 * abs(lb)
    assert np.array_equal(a.topics(), out)


def test_async_host_sweeps_match_resident():
    """lda_iterate_host_async chained through two pinned buffers (each chunk of the next
    input goes up once the previous sweep has brought it down) equals resident sweeps; a
    call after other work on the trainer takes the unchained path and equals the
    synchronous host sweeps; pageable buffers are refused."""
    import torch
    c = L.Corpus.generate(L.corpus_config("c0", num_chunks=4))
    ref = L.Trainer(c, K=64)
    tr = L.Trainer(c, K=64)
    z0 = c.topics()
    pin = lambda a: torch.from_numpy(a.view(np.int16).copy()).pin_memory()
    p, q = pin(z0), pin(np.zeros_like(z0))
    for _ in range(5):
        tr.iterate_host_async(p.numpy().view(np.uint16), q.numpy().view(np.uint16))
        p, q = q, p
    tr.wait()
    ref.iterate(5)
    assert np.array_equal(p.numpy().view(np.uint16), ref.topics())
    assert np.array_equal(tr.topics(), ref.topics())
    # the same calls with other work in between: async, resident sweep, async again from
    # the last output, against the synchronous host path
    s1, s2 = L.Trainer(c, K=64), L.Trainer(c, K=64)
    a1, b1 = pin(z0), pin(np.zeros_like(z0))
    s1.iterate_host_async(a1.numpy().view(np.uint16), b1.numpy().view(np.uint16))
    s1.iterate(1)
    s1.iterate_host_async(b1.numpy().view(np.uint16), a1.numpy().view(np.uint16))
    s1.wait()
    o1, o2 = np.empty_like(z0), np.empty_like(z0)
    s2.iterate_host(z0, o1)
    s2.iterate(1)
    s2.iterate_host(o1, o2)
    assert np.array_equal(a1.numpy().view(np.uint16), o2)
    with pytest.raises(L.LdaError):
        s1.iterate_host_async(z0, np.empty_like(z0))
    # chunks streamed through two slot buffers take the same path
    st = L.Trainer(c, K=64, stream_mode=2, num_streams=2)
    p, q = pin(z0), pin(np.zeros_like(z0))
    for _ in range(3):
        st.iterate_host_async(p.numpy().view(np.uint16), q.numpy().view(np.uint16))
        p, q = q, p
    st.wait()
    ref3 = L.Trainer(c, K=64)
    ref3.iterate(3)
    assert np.array_equal(p.numpy().view(np.uint16), ref3.topics())


def test_checkpoint_resume_is_exact(tmp_path):
    c = L.Corpus.generate(L.corpus_config("c0"))
    a = L.Trainer(c, K=64)
    a.iterate(5)
    p = str(tmp_path / "ck.bin")
    a.checkpoint(p)
    a.iterate(5)
    b = L.Trainer(c, K=64, seed=999)
    b.restore(p)
    assert b.iteration == 5
    b.iterate(5)
    assert np.array_equal(a.topics(), b.topics())


def test_device_budget_and_topic_validation():
    c = L.Corpus.generate(L.corpus_config("c0"))
    with pytest.raises(L.LdaError) as e:
        L.Trainer(c, K=64, device_budget=1 << 16)
    assert e.value.code == -5  # LDA_ERR_DEVICE_MEM
    tr = L.Trainer(c, K=64)
    bad = c.topics()
    bad[3] = 64
    with pytest.raises(L.LdaError) as e:
        tr.set_topics(bad)
    assert e.value.code == -1
    with pytest.raises(L.LdaError) as e:
        tr.perplexity()  # no chunk sampled with ll
    assert e.value.code == -7


def _row_sums(off, ent):
    rows = np.repeat(np.arange(len(off) - 1), np.diff(off))
    return np.bincount(rows, weights=(ent & 0xFFFF).astype(np.float64), minlength=len(off) - 1).astype(np.int64)


@pytest.mark.slow
def test_config1_full_size_properties():
    """Config 1 at full size (K=1024, ~72M tokens): count invariants, determinism, and
    token-for-token agreement with the oracle on every 97th word."""
    c = L.Corpus.generate(L.corpus_config("c1"))
    i = c.info
    K = 1024
    tr = L.Trainer(c, K=K)
    z0 = c.topics()
    tr.update_wt()
    tr.max_topic()
    for ch in range(i.num_chunks):
        tr.update_dt(ch)
    tr.sync()
    nk = tr.topic_totals()
    assert nk.sum() == i.num_tokens and np.array_equal(nk, np.bincount(z0, minlength=K))
    wc = c.word_count()
    assert np.array_equal(tr.dense_wt().sum(1), wc[: i.num_dense])
    soff, sent = tr.sparse_wt()
    assert np.array_equal(_row_sums(soff, sent), wc[i.num_dense:])
    goff, gent = tr.doc_rows()
    assert np.array_equal(_row_sums(goff, gent), np.diff(c.doc_off()))
    for ch in range(i.num_chunks):
        tr.sample_chunk(ch, ll=True)
    ll = tr.perplexity()
    tr.end_sweep()
    z1 = tr.topics()
    assert np.isfinite(ll) and z1.max() < K
    o = Oracle(c.tok_word(), c.tok_doc(), i.vocab, i.num_docs, K, tr.alpha, tr.beta, num_dense=i.num_dense)
    o.rebuild(z0)
    zo = z0.copy()
    st = o.sample(zo, 42, 0, word_stride=97)
    tw = c.tok_word()
    sel = (tw % 97) == 0
    assert st.tokens == sel.sum()
    assert np.array_equal(z1[sel], zo[sel])
    # determinism: a second trainer reproduces the sweep exactly
    tr2 = L.Trainer(c, K=K)
    tr2.iterate(1, ll=True)
    assert np.array_equal(tr2.topics(), z1)
    assert tr2.loglik()[0] == ll


@pytest.mark.parametrize("streams,K", [(1, 64), (2, 64), (3, 64), (2, 4096)])
def test_streamed_chunks_equal_resident(streams, K):
    """Chunks streamed through `streams` slot buffers (EZLDA/mainKernel.cu:203-314) give the
    same topics, LL and counters as the resident corpus, sweep after sweep (K=4096: the
    dense-word and sparse-word samplers of large K)."""
    c = L.Corpus.generate(L.corpus_config("c0", num_chunks=5, dense_kind=1, dense_param=0.05, K=K))
    res = L.Trainer(c, K=K, seed=42, stream_mode=1)
    stm = L.Trainer(c, K=K, seed=42, stream_mode=2, num_streams=streams)
    assert res.stream_info()[0] is False
    on, ns, _ = stm.stream_info()
    assert on and ns == streams
    assert stm.device_bytes < res.device_bytes
    for it in range(6):
        ll_r = res.iterate(1, ll=(it % 2 == 0))
        ll_s = stm.iterate(1, ll=(it % 2 == 0))
        assert np.array_equal(res.topics(), stm.topics()), f"sweep {it}"
        assert ll_r == ll_s
    a, b = res.counters(), stm.counters()
    assert (a.tokens, a.early_accept, a.branch_q) == (b.tokens, b.early_accept, b.branch_q)
    if K <= 2048:
        assert stm.stream_info()[2] == 6 * 12 * c.info.num_tokens
    else:
        # above 2048 topics a chunk that a slot still holds is not copied again
        ct = np.diff(c.chunk_tok())
        copied = _large_k_copies(len(ct), streams, 6)
        assert sum(len(x) for x in copied) < 6 * len(ct)
        assert stm.stream_info()[2] == 12 * sum(int(ct[ch]) for x in copied for ch in x)


def _large_k_copies(n, S, sweeps):
    """The chunks each streamed sweep copies above 2048 topics: sweeps alternate ascending
    and descending chunk order; a chunk no slot holds goes into the slot whose chunk comes
    latest in the rest of the order (never again first), ties to the slot sampled longest
    ago in this sweep, then to the lowest slot."""
    held, down, out = [-1] * S, False, []
    for _ in range(sweeps):
        order = list(range(n))[::-1] if down else list(range(n))
        used, copied = [-1] * S, []
        for i, ch in enumerate(order):
            if ch in held:
                slot = held.index(ch)
            else:
                def nxt(k):
                    h = held[k]
                    pos = order.index(h) if 0 <= h < n else -1
                    return pos if pos > i else n
                slot = max(range(S), key=lambda k: (nxt(k), -used[k]))
                held[slot] = ch
                copied.append(ch)
            used[slot] = i
        out.append(copied)
        down = not down
    return out


def test_streaming_by_budget_and_stage_api():
    """A budget below the resident layout switches to streaming; the stage entry points
    load a chunk in lda_update_dt and refuse to sample a chunk that is not loaded."""
    c = L.Corpus.generate(L.corpus_config("c0", num_chunks=4))
    K = 64
    res = L.Trainer(c, K=K, seed=42)
    full = res.device_bytes
    stm = L.Trainer(c, K=K, seed=42, device_budget=full - 1, num_streams=2)
    assert stm.stream_info()[0]
    assert stm.device_bytes <= full - 1
    o = Oracle(c.tok_word(), c.tok_doc(), c.info.vocab, c.info.num_docs, K, stm.alpha, stm.beta,
               num_dense=c.info.num_dense)
    z = c.topics()
    o.iterate(z, 42, 0)
    stm.update_wt()
    stm.max_topic()
    with pytest.raises(L.LdaError):
        stm.sample_chunk(1)
    for ch in range(c.info.num_chunks):
        stm.update_dt(ch)
        stm.sample_chunk(ch)
    stm.end_sweep()
    assert np.array_equal(stm.topics(), z)
    with pytest.raises(L.LdaError):
        stm.doc_rows()


def test_trainers_of_different_k_coexist():
    """A trainer created after another with a larger K must not lower the kernels' shared
    memory limit below what the first one launches with."""
    big = L.Trainer(L.Corpus.generate(L.corpus_config("c0", num_docs=200, vocab=500, K=1024)), K=1024)
    small = L.Trainer(L.Corpus.generate(L.corpus_config("c0", num_docs=200, vocab=500, K=16)), K=16)
    big.iterate(2, ll=True)
    small.iterate(2, ll=True)
    big.iterate(1)


@pytest.mark.parametrize("stream_mode,chunk_range", [(1, None), (1, (1, 3)), (2, None)])
def test_host_iterate_pinned_buffers(stream_mode, chunk_range):
    """With pinned host buffers each chunk's topics are copied back as soon as the chunk is
    sampled (overlapping the later chunks); the result equals resident sweeps, and tokens
    outside a sampled chunk range come back unchanged."""
    import torch
    c = L.Corpus.generate(L.corpus_config("c0", num_chunks=4))
    a = L.Trainer(c, K=64, stream_mode=1)
    b = L.Trainer(c, K=64, stream_mode=stream_mode, num_streams=2)
    if chunk_range:
        a.set_chunk_range(*chunk_range)
        b.set_chunk_range(*chunk_range)
    z = c.topics()
    zin = torch.empty(len(z), dtype=torch.int16).pin_memory().numpy().view(np.uint16)
    zout = torch.empty(len(z), dtype=torch.int16).pin_memory().numpy().view(np.uint16)
    zin[:] = z
    for it in range(3):
        b.iterate_host(zin, zout)
        a.iterate(1)
        assert np.array_equal(a.topics(), zout), f"sweep {it}"
        zin[:] = zout
    if chunk_range:
        t0, t1 = (int(x) for x in c.chunk_tok()[list(chunk_range)])
        assert np.array_equal(zout[:t0], z[:t0]) and np.array_equal(zout[t1:], z[t1:])


@pytest.mark.parametrize("dense_kind,dense_param", [(0, 0.0), (1, 0.05)])
def test_large_k_word_stats_bit_exact(dense_kind, dense_param):
    """Above 2048 topics sparse words get their statistics without a column (own topics
    plus the CTA's order of beta * r_k); they must equal the oracle's column-based ones."""
    K = 4096
    c = L.Corpus.generate(L.corpus_config("c0", num_docs=400, vocab=900, K=K, num_chunks=2,
                                          dense_kind=dense_kind, dense_param=dense_param))
    tr, o = _setup(c, K)
    tr.iterate(2)
    z = tr.topics()
    o.rebuild(z)
    tr.update_wt()
    tr.max_topic()
    tr.sync()
    for a, b, n in zip(tr.word_stats(), o.word_stats(), ("top2", "k3", "phi4", "ql")):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), n


def test_large_k_word_stats_fallback_scan():
    """A sparse word holding every topic at the head of the beta * r_k order (the topics
    with the fewest tokens) makes the statistics fall back to scanning all topics."""
    K = 4096
    # word "a": one token on each of topics 0..99; word "b": two tokens on every other topic
    wa = [0] * 100
    ta = list(range(100))
    wb = [1] * (2 * (K - 100))
    tb = [k for k in range(100, K) for _ in range(2)]
    words = np.array(wa + wb, dtype=np.int32)
    topics = np.array(ta + tb, dtype=np.uint16)
    doc_off = np.arange(0, len(words) + 1, 400, dtype=np.int64)
    doc_off[-1] = len(words)
    if doc_off[-2] == doc_off[-1]:
        doc_off = doc_off[:-1]
    c = L.Corpus.from_docs(doc_off, words, vocab=2, K=K, topics=topics, num_chunks=1)
    tr, o = _setup(c, K)
    o.rebuild(c.topics())
    tr.update_wt()
    tr.max_topic()
    tr.sync()
    assert c.info.num_dense == 1
    for a, b, n in zip(tr.word_stats(), o.word_stats(), ("top2", "k3", "phi4", "ql")):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), n
