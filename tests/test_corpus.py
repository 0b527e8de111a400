"""CPU tests of the corpus layout, the synthetic generator and the EZLDA chunk format."""
import os

import numpy as np
import pytest

import lda_sc20_b200 as L
from lda_sc20_b200 import LdaError
from oracle import Oracle


def _gen(**over):
    return L.Corpus.generate(L.corpus_config("c0", **over))


def _check_layout(c):
    i = c.info
    tw, td, z = c.tok_word(), c.tok_doc(), c.topics()
    doc_off, pos, dw = c.doc_off(), c.dtok_pos(), c.dtok_word()
    ct, cd = c.chunk_tok(), c.chunk_doc()
    so, sc = c.seg_off(), c.seg_cnt()
    N = i.num_tokens
    assert doc_off[0] == 0 and doc_off[-1] == N
    assert ct[0] == 0 and ct[-1] == N and cd[0] == 0 and cd[-1] == i.num_docs
    assert np.array_equal(np.sort(pos), np.arange(N))           # doc order -> word-sorted is a permutation
    assert np.array_equal(tw[pos], dw)
    doc_of_j = np.repeat(np.arange(i.num_docs), np.diff(doc_off))
    assert np.array_equal(td[pos], doc_of_j)
    for ch in range(i.num_chunks):
        a, b = ct[ch], ct[ch + 1]
        assert np.all(np.diff(tw[a:b]) >= 0)                    # word-sorted inside the chunk
        assert np.all((td[a:b] >= cd[ch]) & (td[a:b] < cd[ch + 1]))
        same = np.diff(tw[a:b]) == 0
        assert np.all(np.diff(td[a:b])[same] >= 0)              # stable: doc order inside a word
        nz = sc[ch] > 0
        assert np.all(tw[so[ch][nz]] == np.nonzero(nz)[0])
        assert sc[ch].sum() == b - a
    wc = c.word_count()
    assert np.all(np.diff(wc) <= 0)                             # ranks by descending frequency
    assert np.array_equal(np.bincount(tw, minlength=i.vocab), wc)
    assert i.num_dense == 0 or wc[i.num_dense - 1] >= 0
    return tw, td, z


def test_generator_is_deterministic_and_layout_valid():
    a, b = _gen(num_chunks=3), _gen(num_chunks=3)
    ta, tb = _check_layout(a), _check_layout(b)
    for x, y in zip(ta, tb):
        assert np.array_equal(x, y)
    c = _gen(num_chunks=3, corpus_seed=1234)
    assert not np.array_equal(c.tok_word()[:1000], a.tok_word()[:1000])


def test_initial_topics_are_philox():
    c = _gen()
    z = c.topics()
    for t in range(0, len(z), 1013):
        assert z[t] == Oracle.init_topic(42, t, 64)


def test_dense_rule_reference_threshold():
    c = _gen()  # dense_kind 0: count >= K (preprocess/streamTestBalance.cpp:100,291)
    wc, nd = c.word_count(), c.info.num_dense
    assert np.all(wc[:nd] >= 64) and np.all(wc[nd:] < 64)
    c2 = _gen(dense_kind=1, dense_param=0.02)
    assert c2.info.num_dense == 100


def test_ezlda_format_round_trip(tmp_path):
    c = _gen(num_chunks=4)
    d = str(tmp_path / "corpus")
    c.write_ezlda(d, 64)
    for f in ["lengthVec.txt", "docLength.txt", "TLLength.txt", "DTLength.txt", "WTLength.txt", "TLSplit.txt",
              "WTCountOffset.txt"]:
        assert os.path.exists(os.path.join(d, f)), f
    for f in ["TL.txt", "word2DocMap.txt", "doc2WordMap.txt", "wordCountOffset.txt", "docCountOffset.txt",
              "DTCountOffset.txt", "WTCountOffset.txt"]:
        assert os.path.exists(os.path.join(d, "chunk0", f)), f
    r = L.Corpus.load_ezlda(d)
    i, j = c.info, r.info
    assert (i.num_tokens, i.vocab, i.num_docs, i.num_chunks, i.num_dense) == \
           (j.num_tokens, j.vocab, j.num_docs, j.num_chunks, j.num_dense)
    for get in ("tok_word", "tok_doc", "topics", "doc_off", "dtok_pos", "dtok_word", "chunk_tok", "chunk_doc",
                "word_count", "seg_off", "seg_cnt"):
        assert np.array_equal(getattr(c, get)(), getattr(r, get)()), get
    # lengthVec: maxTL maxDT maxWT maxDocs W maxChunkWT numOfWordD numOfWordS
    lv = [int(x) for x in open(os.path.join(d, "lengthVec.txt")).read().split()]
    assert lv[0] == int(np.diff(c.chunk_tok()).max()) and lv[4] == i.vocab
    assert lv[6] == i.num_dense and lv[6] + lv[7] == i.vocab
    tl = np.loadtxt(os.path.join(d, "chunk1", "TL.txt"), dtype=np.int64)
    ct = c.chunk_tok()
    assert np.array_equal(tl, c.topics()[ct[1]:ct[2]].astype(np.int64) + 1)  # 1-based topics on disk
    dtco = np.loadtxt(os.path.join(d, "chunk0", "DTCountOffset.txt"), dtype=np.int64)
    lens = np.diff(c.doc_off())[: len(dtco)]
    assert np.array_equal(dtco[:, 0], np.minimum(((lens - 1) // 32 + 1) * 32, 64))


def test_load_errors(tmp_path):
    c = _gen(num_chunks=2)
    d = str(tmp_path / "c")
    c.write_ezlda(d, 64)
    with pytest.raises(LdaError) as e:
        L.Corpus.load_ezlda(str(tmp_path / "missing"))
    assert e.value.code == -2  # LDA_ERR_IO
    # truncated token list
    p = os.path.join(d, "chunk1", "TL.txt")
    lines = open(p).read().split("\n")
    open(p, "w").write("\n".join(lines[: len(lines) // 2]))
    with pytest.raises(LdaError) as e:
        L.Corpus.load_ezlda(d)
    assert e.value.code == -3  # LDA_ERR_FORMAT
    assert "TL.txt" in str(e.value)
    # map that is not a permutation
    c.write_ezlda(d, 64)
    p = os.path.join(d, "chunk0", "word2DocMap.txt")
    m = open(p).read().split("\n")
    m[1] = m[0]
    open(p, "w").write("\n".join(m))
    with pytest.raises(LdaError) as e:
        L.Corpus.load_ezlda(d)
    assert e.value.code == -3
    # topic out of range
    c.write_ezlda(d, 64)
    p = os.path.join(d, "chunk0", "TL.txt")
    t = open(p).read().split("\n")
    t[0] = "0"
    open(p, "w").write("\n".join(t))
    with pytest.raises(LdaError):
        L.Corpus.load_ezlda(d)
    # missing per-chunk file
    c.write_ezlda(d, 64)
    os.remove(os.path.join(d, "chunk1", "docCountOffset.txt"))
    with pytest.raises(LdaError) as e:
        L.Corpus.load_ezlda(d)
    assert e.value.code == -2


def test_from_docs_and_argument_checks():
    rng = np.random.default_rng(0)
    lens = rng.integers(1, 50, size=40)
    lens[5] = 0  # an empty doc
    off = np.concatenate([[0], np.cumsum(lens)])
    words = rng.integers(0, 30, size=off[-1]).astype(np.int32)
    c = L.Corpus.from_docs(off, words, vocab=30, K=8, num_chunks=2)
    _check_layout(c)
    with pytest.raises(LdaError):
        L.Corpus.from_docs(off, np.full(off[-1], 99, np.int32), vocab=30, K=8)
    bad = L.corpus_config("c0", len_min=0)
    with pytest.raises(LdaError):
        L.Corpus.generate(bad)
    with pytest.raises(LdaError):
        L.Corpus.generate(L.corpus_config("c0", K=70000))


def test_generate_requests_follow_the_corpus_process():
    """Held-out requests: deterministic per seed, lengths clipped, words drawn from the
    corpus' own topic-word distributions (their frequencies track the corpus ranks)."""
    import math
    c = L.Corpus.generate(L.corpus_config("c0"))
    off, w = c.generate_requests(3000, seed=9, len_median=150, len_sigma=1.0, len_min=5, len_max=400)
    off2, w2 = c.generate_requests(3000, seed=9, len_median=150, len_sigma=1.0, len_min=5, len_max=400)
    assert np.array_equal(off, off2) and np.array_equal(w, w2)
    lens = np.diff(off)
    assert lens.min() >= 5 and lens.max() <= 400
    assert abs(math.log(np.median(lens)) - math.log(150)) < 0.1
    assert w.min() >= 0 and w.max() < c.info.vocab
    f_req = np.bincount(w, minlength=c.info.vocab).astype(np.float64)
    f_cor = c.word_count().astype(np.float64)
    top = slice(0, 200)
    r = np.corrcoef(f_req[top], f_cor[top])[0, 1]
    assert r > 0.9, r
    off3, _ = c.generate_requests(10, seed=10)
    assert not np.array_equal(off3, off[:11])
    with pytest.raises(L.LdaError):
        c.generate_requests(3, seed=1, len_min=0)


def test_urn_form_matches_explicit_dirichlet():
    """phi_kind 2 (Polya urn, phi integrated out) and phi_kind 1 (explicit Dirichlet draws)
    are the same generative process: their rank-frequency curves agree."""
    covs = {}
    for kind in (1, 2):
        cov = []
        for seed in (11, 12, 13):
            c = L.Corpus.generate(L.corpus_config("c0", num_docs=1500, vocab=4000, gen_topics=16, phi_kind=kind,
                                                  phi_conc=0.05, phi_zipf_s=1.05, corpus_seed=seed))
            wc = np.sort(c.word_count())[::-1].astype(np.float64)
            tot = wc.sum()
            cov.append([wc[:10].sum() / tot, wc[:100].sum() / tot, wc[:1000].sum() / tot, (wc > 0).mean()])
        covs[kind] = np.mean(cov, axis=0)
    assert np.allclose(covs[1], covs[2], rtol=0.08, atol=0.01), covs
