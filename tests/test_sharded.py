"""Document-sharded sweeps: the exchange on CPU with gloo (world size 2), real sharded
sweeps of the oracle through that exchange on two CPU ranks, and the sharded algorithm on
one GPU with two trainers standing in for two ranks."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

import lda_sc20_b200 as L
from lda_sc20_b200.sharded import (TopicExchange, WordExchange, shard_chunks, shard_words, word_bytes,
                                   word_ranges)


def test_shard_chunks():
    assert shard_chunks(8, 1) == [(0, 8)]
    assert shard_chunks(8, 2) == [(0, 4), (4, 8)]
    assert shard_chunks(8, 3) == [(0, 2), (2, 5), (5, 8)]
    assert shard_chunks(8, 8) == [(i, i + 1) for i in range(8)]
    with pytest.raises(ValueError):
        shard_chunks(2, 3)


def test_shard_words_covers_the_vocabulary_in_order():
    rng = np.random.default_rng(0)
    for V, world in [(1, 1), (10, 3), (1000, 8), (5, 8), (0, 2)]:
        cost = rng.pareto(1.0, size=V) + 0.01
        r = shard_words(cost, world)
        assert len(r) == world and r[0][0] == 0 and r[-1][1] == V
        assert all(a <= b for a, b in r) and all(r[i][1] == r[i + 1][0] for i in range(world - 1))
    # equal costs split evenly; one heavy word takes a share by itself
    assert shard_words(np.ones(12), 4) == [(0, 3), (3, 6), (6, 9), (9, 12)]
    assert (0, 1) in shard_words(np.array([90.0] + [1.0] * 30), 3)
    assert list(word_bytes(4, 2, 16, np.array([3, 1]))) == [64 + 152, 64 + 152, 16 + 152, 8 + 152]


def test_word_ranges_beat_pure_token_and_pure_byte_splits():
    """The planned split's modelled time (max rebuild + all-gather) is no worse than
    balancing tokens alone or bytes alone, on a Zipf vocabulary with a dense head."""
    K, world, Vd = 1024, 8, 2000
    tok = np.maximum(1, (5e6 / np.arange(1, 100001) ** 1.05)).astype(np.int64)
    slot = np.minimum(K, tok[Vd:])
    r, t = word_ranges(tok, Vd, K, slot, world)
    assert r[0][0] == 0 and r[-1][1] == len(tok) and all(r[i][1] == r[i + 1][0] for i in range(world - 1))
    byt = word_bytes(len(tok), Vd, K, slot)

    def model(rr):
        return (max(tok[a:b].sum() for a, b in rr) * 9.0e-12
                + (world - 1) * max(byt[a:b].sum() for a, b in rr) / 770e9)
    assert abs(model(r) - t) <= 1e-9 * t
    assert t <= model(shard_words(tok, world)) + 1e-15 and t <= model(shard_words(byt, world)) + 1e-15


def _word_side(word_tokens, z_by_word, K, Vd, words):
    """The word side of `words` (the rest zero), built with numpy as the trainer lays it
    out: dense rows, sparse rows (k << 16 | count, ascending k) in fixed slots, n_k over
    `words`' tokens, and stand-in statistics that are a function of the word."""
    V = len(word_tokens)
    slot = np.minimum(K, word_tokens[Vd:])
    off = np.concatenate([[0], np.cumsum(slot)]).astype(np.int64)
    n_k = np.zeros(K, np.int32)
    dense = np.zeros((Vd, K), np.int32)
    ent = np.zeros(max(int(off[-1]), 1), np.uint32)
    nnz = np.zeros(V - Vd, np.uint32)
    top2 = np.zeros(V, np.uint32)
    k3 = np.zeros(V, np.uint32)
    phi4 = np.zeros((V, 4), np.float32)
    ql = np.zeros((V, 32), np.float32)
    for w in words:
        h = np.bincount(z_by_word[w], minlength=K).astype(np.int32)
        n_k += h
        if w < Vd:
            dense[w] = h
        else:
            ks = np.nonzero(h)[0]
            s = w - Vd
            ent[off[s]:off[s] + len(ks)] = (ks.astype(np.uint32) << 16) | h[ks].astype(np.uint32)
            nnz[s] = len(ks)
        top2[w], k3[w] = 3 * w + 1, 5 * w + 2
        phi4[w] = w + np.arange(4) / 4
        ql[w] = w * 32 + np.arange(32)
    side = {"n_k": n_k, "dense": dense, "sparse_ent": ent, "sparse_nnz": nnz, "top2": top2, "k3": k3,
            "phi4": phi4, "ql": ql}
    return side, off


def _word_worker(rank, world, port, word_tokens, z_by_word, K, Vd, out):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    V = len(word_tokens)
    _, off = _word_side(word_tokens, z_by_word, K, Vd, [])
    ranges, _ = word_ranges(word_tokens, Vd, K, np.diff(off), world)
    side, _ = _word_side(word_tokens, z_by_word, K, Vd, range(*ranges[rank]))
    t = {f: torch.from_numpy(np.ascontiguousarray(a).reshape(-1).view(np.uint8).copy()) for f, a in side.items()}
    t["n_k"] = torch.from_numpy(side["n_k"].copy())
    ex = WordExchange(t, K, Vd, off, ranges)
    ex.reduce_totals()
    for _ in range(2):  # repeatable in place
        ex.exchange()
    out[rank] = ({f: v.numpy().copy() for f, v in t.items()}, ranges)
    dist.destroy_process_group()


def test_word_exchange_gloo_world2():
    """Each rank builds the word side of its word range only; after the n_k all-reduce and
    the all-gather every rank holds the word side of the whole vocabulary."""
    rng = np.random.default_rng(3)
    K, V, Vd = 16, 60, 9
    word_tokens = np.sort(rng.integers(1, 200, size=V))[::-1].copy()
    z_by_word = [rng.integers(0, K, size=n) for n in word_tokens]
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_word_worker, args=(world, port, word_tokens, z_by_word, K, Vd, out), nprocs=world, join=True)
        res = [out[r] for r in range(world)]
    full, _ = _word_side(word_tokens, z_by_word, K, Vd, range(V))
    ranges = res[0][1]
    assert ranges[0][1] > 0 and ranges[1][1] == V and ranges[0][1] < V
    for r in range(world):
        got = res[r][0]
        assert np.array_equal(got["n_k"], full["n_k"])
        for f, a in full.items():
            if f != "n_k":
                assert np.array_equal(got[f], np.ascontiguousarray(a).reshape(-1).view(np.uint8)), (r, f)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, chunk_tok, ranges, out):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    n = int(chunk_tok[-1])
    z = torch.full((n,), -1, dtype=torch.int16)
    a, b = int(chunk_tok[ranges[rank][0]]), int(chunk_tok[ranges[rank][1]])
    z[a:b] = torch.arange(a, b, dtype=torch.int16) % 1000 + 7 * rank  # this rank's sweep result
    ex = TopicExchange(z, chunk_tok, ranges)
    for _ in range(3):  # exchanges are repeatable in place
        ex.exchange()
    out[rank] = z.numpy().copy()
    dist.destroy_process_group()


def test_topic_exchange_gloo_world2():
    """Each rank writes only its chunks' slice; after the exchange every rank holds every
    rank's slice."""
    chunk_tok = np.array([0, 100, 250, 260, 400, 555])
    ranges = shard_chunks(5, 2)
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, chunk_tok, ranges, out), nprocs=world, join=True)
        res = [out[r] for r in range(world)]
    expect = np.empty(555, np.int16)
    for r, (a, b) in enumerate(ranges):
        s, e = chunk_tok[a], chunk_tok[b]
        expect[s:e] = (np.arange(s, e) % 1000 + 7 * r).astype(np.int16)
    for r in range(world):
        assert np.array_equal(res[r], expect)


def _sharded_worker(rank, world, port, params, sweeps, out):
    """One rank of a document-sharded sweep on CPU: the oracle rebuilds the counts from the
    full topic array, samples only this rank's chunks' documents, and the real TopicExchange
    (gloo all-gather) brings in the other ranks' slices."""
    import torch.distributed as dist
    from oracle import Oracle
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    p = dict(params)
    c = L.Corpus.generate(L.corpus_config(p.pop("preset"), **p))
    i = c.info
    ranges = shard_chunks(i.num_chunks, world)
    cd = c.chunk_doc()
    o = Oracle(c.tok_word(), c.tok_doc(), i.vocab, i.num_docs, 64, 50.0 / 64, 0.01, nthreads=2)
    o.set_doc_range(int(cd[ranges[rank][0]]), int(cd[ranges[rank][1]]))
    z = torch.from_numpy(c.topics().view(np.int16).copy())
    ex = TopicExchange(z, c.chunk_tok(), ranges)
    lls = []
    for it in range(sweeps):
        zz = z.numpy().view(np.uint16)
        st = o.iterate(zz, 42, it, ll=True)
        v = torch.tensor([st.loglik, float(st.tokens)], dtype=torch.float64)
        dist.all_reduce(v)
        lls.append(float(v[0]))
        ex.exchange()
    out[rank] = (z.numpy().view(np.uint16).copy(), lls)
    dist.destroy_process_group()


def test_sharded_oracle_sweeps_gloo_world2():
    """Two CPU ranks run real document-sharded sweeps (each samples its half of the chunks,
    then the gloo all-gather exchange) for four sweeps: every rank ends with the topics of
    one process sweeping all chunks, and the summed LL partials equal its LL."""
    from oracle import Oracle
    params = dict(preset="c0", num_docs=600, vocab=1500, num_chunks=4, dense_kind=1, dense_param=0.05)
    sweeps, world = 4, 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_sharded_worker, args=(world, port, params, sweeps, out), nprocs=world, join=True)
        res = [out[r] for r in range(world)]
    p = dict(params)
    c = L.Corpus.generate(L.corpus_config(p.pop("preset"), **p))
    i = c.info
    o = Oracle(c.tok_word(), c.tok_doc(), i.vocab, i.num_docs, 64, 50.0 / 64, 0.01, nthreads=2)
    z = c.topics()
    for it in range(sweeps):
        st = o.iterate(z, 42, it, ll=True)
        for r in range(world):
            assert abs(res[r][1][it] - st.loglik) <= 1e-9 * abs(st.loglik), (r, it)
    for r in range(world):
        assert np.array_equal(res[r][0], z), f"rank {r}: {(res[r][0] != z).sum()} topics differ"


@pytest.mark.gpu
def test_two_shards_on_one_gpu_match_single_trainer():
    """Two trainers each sample half the chunks of one corpus; copying each one's slice
    into the other after every sweep (what the NCCL broadcast does across GPUs) gives
    topics and an LL identical to one trainer sampling all chunks."""
    c = L.Corpus.generate(L.corpus_config("c0", num_chunks=4, dense_kind=1, dense_param=0.05))
    K = 64
    full = L.Trainer(c, K=K)
    shards = [L.Trainer(c, K=K), L.Trainer(c, K=K)]
    ranges = shard_chunks(4, 2)
    for t, (a, b) in zip(shards, ranges):
        t.set_chunk_range(a, b)
    ct = c.chunk_tok()
    for it in range(5):
        full.iterate(1, ll=True)
        lls = []
        for t in shards:
            t.iterate(1, ll=True)
            lls.append(t.loglik())
        z = [t.topics() for t in shards]
        merged = z[0].copy()
        a, b = ct[ranges[1][0]], ct[ranges[1][1]]
        merged[a:b] = z[1][a:b]
        for t in shards:
            t.set_topics(merged)
        assert np.array_equal(merged, full.topics()), f"sweep {it}"
        s = sum(x[0] for x in lls)
        n = sum(x[1] for x in lls)
        fs, fn = full.loglik()
        assert n == fn and abs(s - fs) <= 1e-9 * abs(fs)


@pytest.mark.gpu
@pytest.mark.parametrize("K,over", [(64, dict(num_chunks=4, dense_kind=1, dense_param=0.05)),
                                    (4096, dict(num_docs=1500, vocab=3000, K=4096, num_chunks=4, dense_kind=1,
                                                dense_param=0.05))])
def test_word_and_doc_sharding_on_one_gpu_match_single_trainer(K, over):
    """The full sharded sweep with two trainers standing in for two ranks: each rebuilds
    the word side of its word range, the n_k sum and the word-side all-gather are done by
    copies (WordExchange.pack / unpack), each samples its chunks, and the topic slices are
    swapped.  Topics and LL equal one trainer's at every sweep; at K=4096 the dense and the
    sparse word statistics both run on word ranges."""
    import torch
    from lda_sc20_b200.sharded import word_side_tensors
    c = L.Corpus.generate(L.corpus_config("c0", **over))
    full = L.Trainer(c, K=K)
    shards = [L.Trainer(c, K=K), L.Trainer(c, K=K)]
    ranges = shard_chunks(4, 2)
    sides = [word_side_tensors(t, 0) for t in shards]
    Vd = shards[0].word_side().num_dense
    assert Vd > 0
    off = sides[0][1]
    wr, _ = word_ranges(c.word_count(), Vd, K, np.diff(off), 2)
    assert 0 < wr[0][1] < c.info.vocab
    qb = 256 * shards[0].word_side().qtab_rounds
    assert (qb > 0) == (K > 2048)
    exs = [WordExchange(s, K, Vd, off, wr, qtab_bytes=qb) for s, _ in sides]
    for t, (a, b), w in zip(shards, ranges, wr):
        t.set_chunk_range(a, b)
        t.set_word_range(*w)
    ct = c.chunk_tok()
    for it in range(5):
        # the single trainer's word side of this sweep's starting topics
        full.update_wt()
        full.max_topic()
        full.sync()
        want = (full.topic_totals(), full.dense_wt(), full.sparse_wt(), full.word_stats())
        full.iterate(1, ll=True)
        for t in shards:
            t.update_wt()
        torch.cuda.synchronize()
        nk = sides[0][0]["n_k"] + sides[1][0]["n_k"]
        for s, _ in sides:
            s["n_k"].copy_(nk)
        for t in shards:
            t.max_topic()
        torch.cuda.synchronize()
        recv = torch.cat([exs[r].pack(rank=r, out=torch.zeros(exs[r].seg, dtype=torch.uint8, device="cuda"))
                          for r in range(2)])
        for r in range(2):
            exs[r].unpack(recv, skip=r)
        torch.cuda.synchronize()
        # every shard now holds the whole word side
        for t in shards:
            assert np.array_equal(t.topic_totals(), want[0])
            assert np.array_equal(t.dense_wt(), want[1])
            for x, y in zip(t.sparse_wt(), want[2]):
                assert np.array_equal(x, y)
            for x, y in zip(t.word_stats(), want[3]):
                assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
        lls = []
        for t in shards:
            t.sweep_chunks(ll=True)
            lls.append(t.loglik())
        z = [t.topics() for t in shards]
        merged = z[0].copy()
        a, b = ct[ranges[1][0]], ct[ranges[1][1]]
        merged[a:b] = z[1][a:b]
        for t in shards:
            t.set_topics(merged)
        assert np.array_equal(merged, full.topics()), f"sweep {it}: {(merged != full.topics()).sum()} differ"
        s = sum(x[0] for x in lls)
        n = sum(x[1] for x in lls)
        fs, fn = full.loglik()
        assert n == fn and abs(s - fs) <= 1e-9 * abs(fs), (it, s, fs)


@pytest.mark.gpu
def test_word_range_guards_whole_sweeps():
    """With a word range set, the trainer's own whole sweeps would sample from one rank's
    partial counts, so they are refused (LDA_ERR_STATE); clearing the range (the whole
    vocabulary) makes them run again.  A range outside the vocabulary is an argument
    error."""
    c = L.Corpus.generate(L.corpus_config("c0", num_chunks=2))
    V = c.info.vocab
    tr = L.Trainer(c, K=64)
    tr.set_word_range(0, V // 2)
    with pytest.raises(L.LdaError) as e:
        tr.iterate(1)
    assert e.value.code == -7
    with pytest.raises(L.LdaError) as e:
        tr.set_word_range(0, V + 1)
    assert e.value.code == -1
    tr.set_word_range(0, V)
    tr.iterate(1)
    ws = tr.word_side()
    assert (ws.K, ws.vocab, ws.num_dense) == (64, V, c.info.num_dense) and ws.n_k and ws.top2
