"""CPU tests of the oracle: known answers, count rebuilds against brute force, and the
sampler's distribution against the exact conditional."""
import numpy as np
import pytest

import lda_sc20_b200 as L
from oracle import Oracle, philox4x32_10

# Philox4x32-10 known-answer vectors published with Random123 (Salmon et al., SC'11):
# (counter, key) -> output.
PHILOX_KAT = [
    ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
    ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
    ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
     [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
]


@pytest.mark.parametrize("ctr,key,out", PHILOX_KAT)
def test_philox_kat(ctr, key, out):
    assert list(philox4x32_10(ctr, key)) == out


def test_uniform_and_init_topic_formula():
    # u = (x0 >> 8) * 2^-24 with ctr = {tok, 0, iter, 'LDA1'}; init = (x0*K) >> 32
    for tok, it, seed in [(0, 0, 42), (12345, 7, 42), (2**31 + 5, 99, 2**40 + 3)]:
        x = philox4x32_10([tok & 0xFFFFFFFF, tok >> 32, it, 0x4C444131], [seed & 0xFFFFFFFF, seed >> 32])
        assert Oracle.token_uniform(seed, it, tok) == np.float32((int(x[0]) >> 8) * 2.0**-24)
        y = philox4x32_10([tok & 0xFFFFFFFF, tok >> 32, 0xFFFFFFFF, 0x494E4954], [seed & 0xFFFFFFFF, seed >> 32])
        assert Oracle.init_topic(seed, tok, 1000) == (int(y[0]) * 1000) >> 32


def _small_corpus(D=300, V=400, K=32, chunks=2, seed=7, dense_param=0.0):
    cfg = L.corpus_config("c0", num_docs=D, vocab=V, K=K, num_chunks=chunks, corpus_seed=seed,
                          dense_kind=0 if dense_param == 0 else 1, dense_param=dense_param)
    return L.Corpus.generate(cfg)


def _brute_counts(tw, td, z, V, D, K):
    nwk = np.zeros((V, K), np.int64)
    np.add.at(nwk, (tw, z), 1)
    ndk = np.zeros((D, K), np.int64)
    np.add.at(ndk, (td, z), 1)
    return nwk, ndk, nwk.sum(0)


def test_rebuild_matches_brute_force():
    c = _small_corpus()
    i = c.info
    K = 32
    tw, td, z = c.tok_word(), c.tok_doc(), c.topics()
    o = Oracle(tw, td, i.vocab, i.num_docs, K, 50.0 / K, 0.01, nthreads=3)
    o.rebuild(z)
    nwk, ndk, nk = _brute_counts(tw, td, z.astype(np.int64), i.vocab, i.num_docs, K)
    assert np.array_equal(o.topic_totals(), nk)
    for w in range(0, i.vocab, 37):
        assert np.array_equal(o.word_row(w), nwk[w])
    off, ent = o.doc_rows()
    for d in range(i.num_docs):
        row = ent[off[d]:off[d + 1]]
        ks = row >> 16
        assert np.all(np.diff(ks.astype(np.int64)) > 0)  # ascending k
        dense = np.zeros(K, np.int64)
        dense[ks] = row & 0xFFFF
        assert np.array_equal(dense, ndk[d])
    # word stats: phi = ((float)n + beta) * (1/((float)n_k + V*beta)) in float32
    Vb = np.float32(i.vocab) * np.float32(0.01)
    r = np.float32(1.0) / (nk.astype(np.float32) + Vb)
    assert np.array_equal(o.recip(), r)
    top2, k3, phi4, ql = o.word_stats()
    for w in range(0, i.vocab, 11):
        col = (nwk[w].astype(np.float32) + np.float32(0.01)) * r
        order = sorted(range(K), key=lambda k: (-col[k], k))
        assert top2[w] & 0xFFFF == order[0] and top2[w] >> 16 == order[1] and k3[w] == order[2]
        assert phi4[w, 0] == col[order[0]] and phi4[w, 1] == col[order[1]] and phi4[w, 2] == col[order[2]]
    meta = o.token_meta()
    mk, k2 = top2[tw] & 0xFFFF, top2[tw] >> 16
    assert np.array_equal(meta & 0xFFFF, ndk[td, mk])
    assert np.array_equal(meta >> 16, ndk[td, k2])


def test_sampler_distribution_matches_exact_conditional():
    """Chi-square of oracle draws (over sweep keys) against the FP64 conditional."""
    c = _small_corpus(D=40, V=60, K=16, chunks=1, seed=3)
    i = c.info
    K = 16
    tw, td, z = c.tok_word(), c.tok_doc(), c.topics()
    o = Oracle(tw, td, i.vocab, i.num_docs, K, 50.0 / K, 0.01, nthreads=2)
    o.rebuild(z)
    toks = [0, len(z) // 3, len(z) - 1]
    draws = {t: np.zeros(K, np.int64) for t in toks}
    n = 4000
    zz = z.copy()
    for it in range(n):
        o.sample(zz, 1234, it)
        for t in toks:
            draws[t][zz[t]] += 1
    for t in toks:
        p = o.token_probs(t)
        exp = p * n
        m = exp > 5
        chi2 = (((draws[t] - exp) ** 2)[m] / exp[m]).sum()
        dof = m.sum() - 1
        # 99.9% quantile of chi-square is below dof + 4.5*sqrt(2*dof) + 10 for these dof
        assert chi2 < dof + 4.5 * np.sqrt(2 * dof) + 10, (t, chi2, dof)
        assert draws[t][~m].sum() <= max(20, 3 * exp[~m].sum() + 10)


def test_split_q_distribution_matches_exact_conditional():
    """Above 2048 topics a sparse word draws its Q bucket in two parts (its own topics,
    then the smoothing table).  Chi-square of the oracle's draws over sweep keys against the
    FP64 conditional, with the high-mass topics as their own bins and the rest pooled in
    blocks of 64 topics (alpha = 0.5 gives the Q bucket most of the mass)."""
    K = 4096
    c = L.Corpus.generate(L.corpus_config("c0", num_docs=30, vocab=50, K=K, num_chunks=1, corpus_seed=8,
                                          len_p1=60.0))
    i = c.info
    assert i.num_dense == 0
    tw, td, z = c.tok_word(), c.tok_doc(), c.topics()
    o = Oracle(tw, td, i.vocab, i.num_docs, K, 0.5, 0.01, nthreads=4, num_dense=0)
    o.rebuild(z)
    q = o.word_stats()[3]
    assert (q[:, 2:] == 0).all() and (q[:, 1] > 0).all()  # split statistics {Qw, Qs, 0, ...}
    toks = [0, len(z) // 2, len(z) - 1]
    n = 6000
    draws = {t: np.zeros(K, np.int64) for t in toks}
    zz = z.copy()
    for it in range(n):
        zz[:] = z
        o.sample(zz, 77, it)
        for t in toks:
            draws[t][zz[t]] += 1
    for t in toks:
        p = o.token_probs(t)
        exp = p * n
        big = exp > 20
        blk = np.arange(K) // 64
        obs = np.concatenate([draws[t][big], np.bincount(blk[~big], draws[t][~big], minlength=64)])
        ex = np.concatenate([exp[big], np.bincount(blk[~big], exp[~big], minlength=64)])
        m = ex > 5
        chi2 = (((obs - ex) ** 2)[m] / ex[m]).sum()
        dof = m.sum() - 1
        assert chi2 < dof + 4.5 * np.sqrt(2 * dof) + 10, (t, chi2, dof)


def test_early_accept_is_exact_in_fp64():
    """A token settled by the max-topic bound gets maxK; in FP64 its u is below
    p_max / total, so the full evaluation would also pick maxK (EZLDA/utility.cu:1341-1373)."""
    c = _small_corpus(D=200, V=300, K=32, chunks=1, seed=11)
    i = c.info
    K, alpha = 32, np.float32(50.0 / 32)
    tw, td, z = c.tok_word(), c.tok_doc(), c.topics()
    o = Oracle(tw, td, i.vocab, i.num_docs, K, alpha, 0.01, nthreads=2)
    zz = z.copy()
    for it in range(6):  # concentrate topics so the bound fires
        o.iterate(zz, 5, it)
    o.rebuild(zz)
    top2, _, _, _ = o.word_stats()
    out = zz.copy()
    st = o.sample(out, 5, 6)
    assert st.early_accept > 0
    meta = o.token_meta()
    checked = 0
    for t in range(0, len(zz), 7):
        mk = top2[tw[t]] & 0xFFFF
        p = o.token_probs(t)
        u = Oracle.token_uniform(5, 6, t)
        if u < 0.9 * p[mk]:
            assert out[t] == mk
            checked += 1
    assert checked > 0 and meta.shape == zz.shape


def test_loglik_matches_numpy_fp64():
    c = _small_corpus(D=150, V=200, K=16, chunks=1, seed=5)
    i = c.info
    K = 16
    alpha, beta = np.float32(50.0 / K), np.float32(0.01)
    tw, td, z = c.tok_word(), c.tok_doc(), c.topics()
    o = Oracle(tw, td, i.vocab, i.num_docs, K, alpha, beta, nthreads=2)
    o.rebuild(z)
    st = o.sample(z.copy(), 9, 0, ll=True)
    nwk, ndk, nk = _brute_counts(tw, td, z.astype(np.int64), i.vocab, i.num_docs, K)
    phi = (nwk + float(beta)) / (nk + i.vocab * float(beta))
    nd = ndk.sum(1)
    tot = ((ndk[td] + float(alpha)) * phi[tw]).sum(1)
    ll = np.log(tot / (nd[td] + K * float(alpha))).sum()
    assert st.tokens == len(z)
    assert abs(st.loglik - ll) <= 1e-5 * abs(ll)


def test_iterate_is_deterministic_across_thread_counts():
    c = _small_corpus(D=120, V=150, K=16, chunks=1, seed=2)
    i = c.info
    tw, td, z = c.tok_word(), c.tok_doc(), c.topics()
    res = []
    for nt in (1, 4):
        o = Oracle(tw, td, i.vocab, i.num_docs, 16, 50.0 / 16, 0.01, nthreads=nt)
        zz = z.copy()
        lls = [o.iterate(zz, 3, it, ll=True).loglik for it in range(4)]
        res.append((zz, lls))
    assert np.array_equal(res[0][0], res[1][0])
    assert res[0][1] == res[1][1]


def test_foldin_keys_and_theta_formula():
    """Fold-in randoms: u = (x0>>8)*2^-24 with ctr = {pos, rid, sweep, 'FOLD'}; initial
    topics (x0*K)>>32 with ctr = {pos, rid, 0xFFFFFFFF, 'FINI'}; with zero sweeps theta is
    ((float)n_dk + alpha) / ((float)len + (float)K*alpha) of the initial topics."""
    from oracle import lib
    seed, rid, K = 2**33 + 9, 17, 48
    for pos, sw in [(0, 0), (5, 3), (65534, 29)]:
        x = philox4x32_10([pos, rid, sw, 0x464F4C44], [seed & 0xFFFFFFFF, seed >> 32])
        assert lib().orc_foldin_uniform(seed, rid, sw, pos) == np.float32((int(x[0]) >> 8) * 2.0**-24)
        y = philox4x32_10([pos, rid, 0xFFFFFFFF, 0x46494E49], [seed & 0xFFFFFFFF, seed >> 32])
        assert lib().orc_foldin_init(seed, rid, pos, K) == (int(y[0]) * K) >> 32
    c = _small_corpus(D=80, V=120, K=K, chunks=1, seed=5)
    i = c.info
    o = Oracle(c.tok_word(), c.tok_doc(), i.vocab, i.num_docs, K, 50.0 / K, 0.01, nthreads=2)
    o.rebuild(c.topics())
    words = np.arange(37, dtype=np.int32) % i.vocab
    z, th = o.foldin(words, rid, seed, 0)
    assert [int(t) for t in z] == [lib().orc_foldin_init(seed, rid, p, K) for p in range(len(words))]
    a = np.float32(o.alpha)
    h = np.bincount(z, minlength=K).astype(np.float32)
    assert np.array_equal(th, (h + a) / (np.float32(len(words)) + np.float32(K) * a))
    z1, th1 = o.foldin(words, rid, seed, 4)
    z2, th2 = o.foldin(words, rid, seed, 4)
    assert np.array_equal(z1, z2) and np.array_equal(th1, th2)
    with pytest.raises(ValueError):
        o.foldin(np.array([i.vocab], dtype=np.int32), 0, seed, 1)


def test_foldin_draw_matches_exact_conditional():
    """Chi-square of one-sweep fold-in draws of one token (over request ids, each with its
    own initial topics) against the summed FP64 conditionals (n_dk + alpha) * phi_wk of
    the frozen word side."""
    K = 16
    c = _small_corpus(D=60, V=80, K=K, chunks=1, seed=4)
    i = c.info
    o = Oracle(c.tok_word(), c.tok_doc(), i.vocab, i.num_docs, K, 50.0 / K, 0.01, nthreads=2)
    o.rebuild(c.topics())
    words = np.array([3, 3, 10, 41, 7, 3, 55, 10, 0, 79, 12, 3], dtype=np.int32)
    phi = {int(w): o.phi_row(int(w)).astype(np.float64) for w in np.unique(words)}
    n, tok = 3000, 5
    obs = np.zeros(K, np.int64)
    exp = np.zeros(K, np.float64)
    for rid in range(n):
        z0, _ = o.foldin(words, rid, 99, 0)
        z1, _ = o.foldin(words, rid, 99, 1)
        h = np.bincount(z0, minlength=K).astype(np.float64)
        p = (h + o.alpha) * phi[int(words[tok])]
        exp += p / p.sum()
        obs[z1[tok]] += 1
    m = exp > 5
    chi2 = (((obs - exp) ** 2)[m] / exp[m]).sum()
    dof = m.sum() - 1
    assert chi2 < dof + 4.5 * np.sqrt(2 * dof) + 10, (chi2, dof)
