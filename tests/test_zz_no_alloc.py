"""The allocation-free sampling entry point against lda_sample_chunk.

lda_sample_chunk_noalloc serves callers that own all device memory through their own
allocator or a reserved arena and cannot let a library call cudaMalloc/cudaFree (those
calls synchronise the device and can fail mid-request).  This test plays such a caller:
it holds every input and output in its own device buffers (torch tensors), calls the
entry point twice in a row through the C ABI, and checks both calls against the
library's own lda_sample_chunk on the same state: identical topics, LL within 1e-9."""
import ctypes as C

import numpy as np
import pytest

import lda_sc20_b200 as L
from lda_sc20_b200 import _native

pytestmark = pytest.mark.gpu

LL_RTOL = 1e-9
TILE = 4096


def _tiles_for_chunk(corpus, chunk, num_dense):
    so, sc = corpus.seg_off()[chunk], corpus.seg_cnt()[chunk]
    tiles = []
    for w in np.nonzero(sc)[0]:
        for p in range(0, int(sc[w]), TILE):
            tiles.append((int(w), int(so[w]) + p, min(TILE, int(sc[w]) - p), 1 if w < num_dense else 0))
    return np.array(tiles, dtype=np.int32).reshape(-1, 4)


def _aligned_rows(off, ent):
    """Doc rows re-laid so that each row starts at a multiple of 4 entries."""
    nnz = np.diff(off).astype(np.int64)
    cap = (nnz + 3) & ~3
    new_off = np.concatenate([[0], np.cumsum(cap)[:-1]]).astype(np.int64)
    out = np.zeros(max(int(cap.sum()), 4), dtype=np.uint32)
    for d in range(len(nnz)):
        out[new_off[d]:new_off[d] + nnz[d]] = ent[off[d]:off[d + 1]]
    return new_off.astype(np.uint32), nnz.astype(np.uint32), out


def test_noalloc_sampling_matches_sample_chunk():
    torch = pytest.importorskip("torch")
    corpus = L.Corpus.generate(L.corpus_config("c0", num_chunks=1, dense_kind=1, dense_param=0.05))
    info = corpus.info
    K = 64
    tr = L.Trainer(corpus, K=K, seed=42)
    tr.iterate(3)  # a state away from the random start
    z_before = tr.topics()
    it = tr.iteration
    tr.update_wt()
    tr.max_topic()
    tr.update_dt(0)
    tr.sync()
    n_k = tr.topic_totals()
    dwt = tr.dense_wt()
    soff, sent = tr.sparse_wt()
    top2, _, phi4, ql = tr.word_stats()
    doff, dent = tr.doc_rows()
    meta = tr.token_meta()
    # the library's own entry point on the same state
    tr.sample_chunk(0, ll=True)
    ll_ref = tr.perplexity()
    z_ref = tr.topics()

    dev = torch.device("cuda", 0)

    def t(a, dtype=None):
        a = np.ascontiguousarray(a)
        if dtype is not None:
            a = a.view(dtype)
        if a.dtype == np.uint32:
            a = a.view(np.int32)
        if a.dtype == np.uint16:
            a = a.view(np.int16)
        return torch.from_numpy(a.copy()).to(dev)

    tiles = _tiles_for_chunk(corpus, 0, info.num_dense)
    dt_off, dt_nnz, dt_ent = _aligned_rows(doff, dent)
    bufs = dict(
        tiles=t(tiles.reshape(-1)), n_k=t(n_k), dense_wt=t(dwt.reshape(-1) if dwt.size else np.zeros(4, np.int32)),
        sparse_off=t(soff[:-1].astype(np.uint32)), sparse_nnz=t(np.diff(soff).astype(np.uint32)),
        sparse_ent=t(sent if len(sent) else np.zeros(4, np.uint32)), top2=t(top2), phi4=t(phi4.reshape(-1)),
        ql=t(ql.reshape(-1)), tok_doc=t(corpus.tok_doc()), meta=t(meta),
        doc_len=t(np.diff(corpus.doc_off()).astype(np.uint32)), dt_off=t(dt_off), dt_nnz=t(dt_nnz),
        dt_ent=t(dt_ent))
    ll_out = torch.zeros(1, dtype=torch.float64, device=dev)
    lib = _native.load()
    for call in range(2):
        topics = t(z_before)
        ll_out.zero_()
        io = _native.SampleIO(K=K, num_dense=info.num_dense, vocab=info.vocab, alpha=tr.alpha, beta=tr.beta,
                              seed=42, iter=it, ll_mode=1, num_tiles=len(tiles),
                              topics=topics.data_ptr(), ll_sum=ll_out.data_ptr(),
                              **{k: v.data_ptr() for k, v in bufs.items()})
        _native.check(lib.lda_sample_chunk_noalloc(C.byref(io), 0, None))
        torch.cuda.synchronize()
        got = topics.cpu().numpy().view(np.uint16)
        assert np.array_equal(got, z_ref), f"call {call}: {(got != z_ref).sum()} topics differ"
        ll = float(ll_out.item())
        assert abs(ll - ll_ref) <= LL_RTOL * abs(ll_ref), (call, ll, ll_ref)


def test_noalloc_rejects_too_many_tiles():
    io = _native.SampleIO(K=64, num_dense=0, vocab=10, alpha=0.5, beta=0.01, num_tiles=65537)
    with pytest.raises(L.LdaError) as e:
        _native.check(_native.load().lda_sample_chunk_noalloc(C.byref(io), 0, None))
    assert e.value.code == -1 and "65536" in str(e.value)
