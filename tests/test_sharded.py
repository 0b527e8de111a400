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
from lda_sc20_b200.sharded import TopicExchange, shard_chunks


def test_shard_chunks():
    assert shard_chunks(8, 1) == [(0, 8)]
    assert shard_chunks(8, 2) == [(0, 4), (4, 8)]
    assert shard_chunks(8, 3) == [(0, 2), (2, 5), (5, 8)]
    assert shard_chunks(8, 8) == [(i, i + 1) for i in range(8)]
    with pytest.raises(ValueError):
        shard_chunks(2, 3)


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
