"""The allocation-free sampling entry point against lda_sample_chunk.

lda_sample_chunk_noalloc serves callers that own all device memory through their own
allocator or a reserved arena and cannot let a library call cudaMalloc/cudaFree (those
calls synchronise the device and can fail mid-request).  These tests play such a caller:
every input and output sits in the test's own device buffers (torch tensors), the entry
point is called twice in a row through the C ABI, and both calls are checked against the
library's own lda_sample_chunk on the same state: identical topics, LL within 1e-9.
K=64 and K=1024 run the per-warp-column sampler the trainer also uses; at K=4096 the
trainer splits dense and sparse words over its two large-K kernels while this entry point
uses the per-warp-column one, and the topics must still agree.  A planted out-of-range
topic must be caught by the device-side checks before any token is sampled."""
import ctypes as C

import numpy as np
import pytest

import lda_sc20_b200 as L
from lda_sc20_b200 import _native

pytestmark = pytest.mark.gpu

LL_RTOL = 1e-9
TILE = 4096
IO_DOC_ROW = 16  # LDA_IO_DOC_ROW


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


def _state(K, cfg):
    """A one-chunk trainer three sweeps in, its sweep-start state for the next sweep, and
    that sweep's topics and LL from lda_sample_chunk."""
    corpus = L.Corpus.generate(cfg)
    tr = L.Trainer(corpus, K=K, seed=42)
    tr.iterate(3)
    st = {"corpus": corpus, "tr": tr, "z_before": tr.topics(), "iter": tr.iteration}
    tr.update_wt()
    tr.max_topic()
    tr.update_dt(0)
    tr.sync()
    st.update(n_k=tr.topic_totals(), dwt=tr.dense_wt(), swt=tr.sparse_wt(), stats=tr.word_stats(),
              rows=tr.doc_rows(), meta=tr.token_meta())
    tr.sample_chunk(0, ll=True)
    st["ll_ref"] = tr.perplexity()
    st["z_ref"] = tr.topics()
    return st


def _device_io(torch, st, K):
    dev = torch.device("cuda", 0)
    corpus, tr = st["corpus"], st["tr"]
    info = corpus.info

    def t(a):
        a = np.ascontiguousarray(a)
        if a.dtype == np.uint32:
            a = a.view(np.int32)
        if a.dtype == np.uint16:
            a = a.view(np.int16)
        return torch.from_numpy(a.copy()).to(dev)

    tiles = _tiles_for_chunk(corpus, 0, info.num_dense)
    dt_off, dt_nnz, dt_ent = _aligned_rows(*st["rows"])
    soff, sent = st["swt"]
    top2, _, phi4, ql = st["stats"]
    dwt = st["dwt"]
    bufs = dict(
        tiles=t(tiles.reshape(-1)), n_k=t(st["n_k"]),
        dense_wt=t(dwt.reshape(-1) if dwt.size else np.zeros(4, np.int32)),
        sparse_off=t(soff[:-1].astype(np.uint32)), sparse_nnz=t(np.diff(soff).astype(np.uint32)),
        sparse_ent=t(sent if len(sent) else np.zeros(4, np.uint32)), top2=t(top2), phi4=t(phi4.reshape(-1)),
        ql=t(ql.reshape(-1)), tok_doc=t(corpus.tok_doc()), meta=t(st["meta"]),
        doc_len=t(np.diff(corpus.doc_off()).astype(np.uint32)), dt_off=t(dt_off), dt_nnz=t(dt_nnz),
        dt_ent=t(dt_ent))
    sizes = dict(num_tokens=info.num_tokens, num_docs=info.num_docs, num_dt_entries=len(dt_ent),
                 num_sparse_entries=max(len(sent), 4))
    return bufs, sizes, len(tiles)


def _call(torch, st, K, bufs, sizes, ntiles):
    dev = torch.device("cuda", 0)
    tr, info = st["tr"], st["corpus"].info
    topics = torch.from_numpy(st["z_before"].view(np.int16).copy()).to(dev)
    ll_out = torch.zeros(1, dtype=torch.float64, device=dev)
    status = torch.full((1,), -1, dtype=torch.int32, device=dev)
    io = _native.SampleIO(K=K, num_dense=info.num_dense, vocab=info.vocab, alpha=tr.alpha, beta=tr.beta,
                          seed=42, iter=st["iter"], ll_mode=1, num_tiles=ntiles,
                          topics=topics.data_ptr(), ll_sum=ll_out.data_ptr(), status=status.data_ptr(),
                          **sizes, **{k: v.data_ptr() for k, v in bufs.items()})
    _native.check(_native.load().lda_sample_chunk_noalloc(C.byref(io), 0, None))
    torch.cuda.synchronize()
    return topics.cpu().numpy().view(np.uint16), float(ll_out.item()), int(status.item())


CASES = {
    64: dict(preset="c0", num_chunks=1, dense_kind=1, dense_param=0.05),
    1024: dict(preset="c0", num_docs=1500, vocab=3000, K=1024, num_chunks=1, dense_kind=1, dense_param=0.05),
    4096: dict(preset="c0", num_docs=1500, vocab=3000, K=4096, num_chunks=1, dense_kind=1, dense_param=0.05),
}


@pytest.mark.parametrize("K", sorted(CASES))
def test_noalloc_sampling_matches_sample_chunk(K):
    torch = pytest.importorskip("torch")
    p = dict(CASES[K])
    cfg = L.corpus_config(p.pop("preset"), **p)
    st = _state(K, cfg)
    assert st["corpus"].info.num_dense > 0
    bufs, sizes, ntiles = _device_io(torch, st, K)
    for call in range(2):
        got, ll, status = _call(torch, st, K, bufs, sizes, ntiles)
        assert status == 0, f"call {call}: device checks failed ({status})"
        assert np.array_equal(got, st["z_ref"]), f"call {call}: {(got != st['z_ref']).sum()} topics differ"
        assert abs(ll - st["ll_ref"]) <= LL_RTOL * abs(st["ll_ref"]), (call, ll, st["ll_ref"])


def test_noalloc_checks_reject_an_out_of_range_row_topic():
    """A doc-row topic of K (one past the last) is reported in the status word and no
    token is sampled; the next call with the row repaired samples as lda_sample_chunk.
    (At K=64 the skewed word column has padding slots past topic K-1, so even an unchecked
    read of topic K would stay inside the column.)"""
    torch = pytest.importorskip("torch")
    K = 64
    p = dict(CASES[K])
    st = _state(K, L.corpus_config(p.pop("preset"), **p))
    bufs, sizes, ntiles = _device_io(torch, st, K)
    good = bufs["dt_ent"].clone()
    ent = good.cpu().numpy().view(np.uint32).copy()
    first = int(np.nonzero(ent)[0][0])
    ent[first] = (np.uint32(K) << 16) | (ent[first] & 0xFFFF)
    bufs["dt_ent"] = torch.from_numpy(ent.view(np.int32)).to(good.device)
    got, _, status = _call(torch, st, K, bufs, sizes, ntiles)
    assert status & IO_DOC_ROW
    assert np.array_equal(got, st["z_before"]), "a rejected call must leave the topics as they were"
    bufs["dt_ent"] = good
    got, _, status = _call(torch, st, K, bufs, sizes, ntiles)
    assert status == 0 and np.array_equal(got, st["z_ref"])


def test_noalloc_rejects_too_many_tiles():
    io = _native.SampleIO(K=64, num_dense=0, vocab=10, alpha=0.5, beta=0.01, num_tiles=65537)
    with pytest.raises(L.LdaError) as e:
        _native.check(_native.load().lda_sample_chunk_noalloc(C.byref(io), 0, None))
    assert e.value.code == -1 and "65536" in str(e.value)
