"""Runs EZLDA's own kernels (oracle/_ref/ref_harness) on seeded corpora and writes the
golden fixtures that pin the oracle to the reference.

TEST INFRASTRUCTURE ONLY.  Needs a GPU and the prebuilt oracle/_ref/ref_harness.

    python oracle/ref/run_ref.py OUTDIR [--modes=counts,sweeps,dist] [--sweeps=100]

Fixtures written to OUTDIR (then committed under tests/golden/):
  ref_counts.npz   the reference's count rebuild and max-topic outputs on corpus
                   REF_COUNTS (dense and sparse words, K=1024): n_k, sparse WT, dense WT,
                   DT rows, per-token doc metadata, per-word max/2nd/3rd topic, phi and Q
  ref_ll.json      the reference's per-sweep log-likelihood curve (computed with the
                   oracle's FP64 LL from the reference's topics) on corpus REF_SWEEPS,
                   over 100 sweeps (EZLDA/mainKernel.cu:51 numIters = 100)
  ref_dist.npz     histograms of the reference sampler's draws for tracked tokens over
                   independent sweeps from one state, corpus REF_DIST
The corpora are regenerated from their generator parameters (stored in each fixture)
by lda_sc20_b200's deterministic generator.
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import lda_sc20_b200 as L  # noqa: E402
from oracle import Oracle  # noqa: E402

HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
K = 1024
ALPHA = np.float32(50.0 / K)  # EZLDA/Argument.cuh:9 (double 50/K passed to the kernels as float)
BETA = np.float32(0.01)

# corpus generator parameters of each fixture (lda_sc20_b200.corpus_config overrides)
REF_COUNTS = dict(preset="c1", num_docs=200, vocab=3000, num_chunks=2, dense_kind=0, corpus_seed=2024)
REF_SWEEPS = dict(preset="c1", num_docs=8000, vocab=20000, phi_kind=0, phi_conc=0.05, num_chunks=8,
                  dense_kind=2, dense_param=0.0, corpus_seed=3030)
# EZLDA's timing on the same B200: the largest corpus shape its sparse path handles
# (every word under K occurrences per chunk, no dense words), K=1024, 8 chunks, ~14.5M tokens
REF_TIME = dict(preset="c1", num_docs=60000, vocab=100000, phi_kind=0, phi_conc=0.05, num_chunks=8,
                dense_kind=2, dense_param=0.0, corpus_seed=5050)
REF_DIST = dict(preset="c0", num_docs=50, vocab=300, K=K, len_p1=50.0, num_chunks=2, dense_kind=2,
                dense_param=0.0, corpus_seed=4040)


def make_corpus(params: dict):
    p = dict(params)
    preset = p.pop("preset")
    return L.Corpus.generate(L.corpus_config(preset, **p))


def run_harness(*args):
    r = subprocess.run([HARNESS] + [str(a) for a in args], capture_output=True, text=True, timeout=1200)
    if r.returncode != 0:
        raise RuntimeError(f"ref_harness {args[0]} failed ({r.returncode}): {r.stderr[-2000:]}")
    return r.stdout


def _rd(path, dtype):
    return np.fromfile(path, dtype=dtype)


def load_counts_dump(d: str, nchunks: int) -> dict:
    out = {n: _rd(os.path.join(d, f), t) for n, f, t in [
        ("nk", "nk.i32", np.int32), ("swt_nnz", "swt_nnz.i32", np.int32), ("swt_idx", "swt_idx.u16", np.uint16),
        ("swt_val", "swt_val.u16", np.uint16), ("wt_off", "wt_off.i32", np.int32), ("dwt", "dwt.i32", np.int32),
        ("wmax", "wmax.u16", np.uint16), ("w2nd", "w2nd.u16", np.uint16), ("w3rd", "w3rd.u16", np.uint16),
        ("pmax", "pmax.f32", np.float32), ("p2nd", "p2nd.f32", np.float32), ("p3rd", "p3rd.f32", np.float32),
        ("qarr", "qarr.f32", np.float32)]}
    for c in range(nchunks):
        for n, t in [("meta", np.int64), ("dt_nnz", np.int32), ("dt_ent", np.int32), ("dt_off", np.int32)]:
            ext = {np.int64: "i64", np.int32: "i32"}[t]
            out[f"c{c}_{n}"] = _rd(os.path.join(d, f"c{c}_{n}.{ext}"), t)
    return out


def compare_counts(corpus, ref: dict) -> dict:
    """Compares the reference's dumps with the oracle on the same topics.  Integer state
    must match exactly; the max topics may differ only between topics whose phi ties."""
    i = corpus.info
    V, Vd = i.vocab, i.num_dense
    o = Oracle(corpus.tok_word(), corpus.tok_doc(), V, i.num_docs, K, ALPHA, BETA)
    z = corpus.topics()
    o.rebuild(z)
    res = {}
    res["n_k"] = bool(np.array_equal(ref["nk"], o.topic_totals()))
    dwt = ref["dwt"].reshape(Vd, K) if Vd else np.zeros((0, K), np.int32)
    res["dense_wt"] = all(np.array_equal(dwt[w], o.word_row(w)) for w in range(Vd))
    ooff, oent = o.word_rows_packed(Vd, V)
    base = int(ref["wt_off"][Vd]) if Vd < V else 0
    ok = True
    for s in range(V - Vd):
        n = int(ref["swt_nnz"][s])
        a = int(ref["wt_off"][Vd + s]) - base
        got = (ref["swt_idx"][a:a + n].astype(np.uint32) - 1) << 16 | ref["swt_val"][a:a + n].astype(np.uint32)
        if not np.array_equal(got, oent[ooff[s]:ooff[s + 1]]):
            ok = False
            break
    res["sparse_wt"] = ok
    roff, rent = o.doc_rows()
    ct, cd = corpus.chunk_tok(), corpus.chunk_doc()
    dt_ok, meta_ok, doc_ok = True, True, True
    top2, k3, phi4, ql = o.word_stats()
    wmax = ref["wmax"].astype(np.int64) - 1
    w2nd = ref["w2nd"].astype(np.int64) - 1
    tw, td = corpus.tok_word(), corpus.tok_doc()
    for c in range(i.num_chunks):
        nnz, ent, off = ref[f"c{c}_dt_nnz"], ref[f"c{c}_dt_ent"], ref[f"c{c}_dt_off"]
        for j in range(int(cd[c + 1] - cd[c])):
            d = int(cd[c]) + j
            got = ent[off[j]:off[j] + nnz[j]].astype(np.int64) - (1 << 16)
            if not np.array_equal(got.astype(np.uint32), rent[roff[d]:roff[d + 1]]):
                dt_ok = False
        meta = ref[f"c{c}_meta"]
        g = np.arange(ct[c], ct[c + 1])
        if not np.array_equal((meta >> 32) - 1 + cd[c], td[g]):
            doc_ok = False
        # the reference's counts of ITS max / 2nd topic of the token's word, recounted
        # from the oracle's doc rows
        for t_local, t in enumerate(g):
            d, w = td[t], tw[t]
            row = rent[roff[d]:roff[d + 1]]
            ks, cs = row >> 16, row & 0xFFFF
            cm = int(cs[ks == wmax[w]].sum())
            c2 = int(cs[ks == w2nd[w]].sum())
            if int(meta[t_local] & 0xFFFFFFFF) != ((c2 << 16) | cm):
                meta_ok = False
                break
    res["doc_rows"] = dt_ok
    res["doc_ids"] = doc_ok
    res["token_meta"] = meta_ok
    # max topics: equal, or the phi of the two choices tie to within 2 ulp
    n_k = o.topic_totals()
    r = np.float32(1.0) / (n_k.astype(np.float32) + np.float32(V) * BETA)
    same_max = same_2nd = same_3rd = 0
    tie_ok = True
    qrel = 0.0
    for w in range(V):
        col = (o.word_row(w).astype(np.float32) + BETA) * r
        ours = [int(top2[w] & 0xFFFF), int(top2[w] >> 16), int(k3[w])]
        refk = [int(wmax[w]), int(w2nd[w]), int(ref["w3rd"][w]) - 1]
        same_max += ours[0] == refk[0]
        same_2nd += ours[1] == refk[1]
        same_3rd += ours[2] == refk[2]
        for a, b in zip(ours, refk):
            if a != b and abs(float(col[a]) - float(col[b])) > 2 * np.spacing(np.float32(col[a])):
                tie_ok = False
        qref = float(ref["qarr"][w])
        qours = float(phi4[w, 3]) / float(ALPHA)
        qrel = max(qrel, abs(qours - qref) / qref)
        pr = float(ref["pmax"][w])
        if abs(pr - float(col[refk[0]])) > 4 * np.spacing(np.float32(pr)):
            tie_ok = False
    res["max_topic_same"] = [same_max, same_2nd, same_3rd, V]
    res["max_topic_ties_only"] = tie_ok
    res["q_max_rel_diff"] = qrel
    return res


def mode_counts(tmp, out):
    c = make_corpus(REF_COUNTS)
    d = os.path.join(tmp, "counts")
    c.write_ezlda(d, K)
    dump = os.path.join(tmp, "counts_out")
    os.makedirs(dump)
    log = run_harness("counts", d, dump)
    ref = load_counts_dump(dump, c.info.num_chunks)
    res = compare_counts(c, ref)
    np.savez_compressed(os.path.join(out, "ref_counts.npz"), params=json.dumps(REF_COUNTS), K=K, **ref)
    return {"log": log.strip(), **res}


def oracle_ll(o: Oracle, z: np.ndarray) -> float:
    o.rebuild(z)
    st = o.sample(z.copy(), 1, 0, ll=True)
    return st.loglik / st.tokens


def mode_sweeps(tmp, out, n=100):
    c = make_corpus(REF_SWEEPS)
    i = c.info
    d = os.path.join(tmp, "sweeps")
    c.write_ezlda(d, K)
    dump = os.path.join(tmp, "sweeps_out")
    os.makedirs(dump)
    log = run_harness("sweeps", d, dump, n)
    o = Oracle(c.tok_word(), c.tok_doc(), i.vocab, i.num_docs, K, ALPHA, BETA)
    z0 = c.topics()
    curve = [oracle_ll(o, z0)]
    for it in range(n):
        z = np.fromfile(os.path.join(dump, f"topics_{it}.u16"), dtype=np.uint16) - 1
        assert len(z) == i.num_tokens and z.max() < K
        curve.append(oracle_ll(o, z.astype(np.uint16)))
    # our sampler from the same initial topics, LL of each state by the same function
    tr = L.Trainer(c, K=K, alpha=float(ALPHA), beta=float(BETA), seed=42)
    ours = [curve[0]]
    for it in range(n):
        tr.iterate(1)
        ours.append(oracle_ll(o, tr.topics()))
    rel = [abs(a - b) / abs(b) for a, b in zip(ours, curve)]
    with open(os.path.join(out, "ref_ll.json"), "w") as f:
        json.dump({"params": REF_SWEEPS, "K": K, "alpha": float(ALPHA), "beta": float(BETA),
                   "ll_per_token_after_sweep": curve, "tokens": i.num_tokens,
                   "note": "index 0 = initial topics; index s = after s reference sweeps"}, f, indent=1)
    return {"log": log.strip(), "ref_curve": curve, "our_curve": ours, "max_rel_diff": max(rel)}


def mode_dist(tmp, out, reps=2000, stride=25):
    from scipy.stats import chi2
    c = make_corpus(REF_DIST)
    i = c.info
    d = os.path.join(tmp, "dist")
    c.write_ezlda(d, K)
    dump = os.path.join(tmp, "dist_out")
    os.makedirs(dump)
    log = run_harness("dist", d, dump, reps, stride)
    tracked = np.fromfile(os.path.join(dump, "dist_tracked.i64"), dtype=np.int64)
    hist = np.fromfile(os.path.join(dump, "dist_hist.i32"), dtype=np.int32).reshape(len(tracked), K)
    o = Oracle(c.tok_word(), c.tok_doc(), i.vocab, i.num_docs, K, ALPHA, BETA)
    o.rebuild(c.topics())
    pvals = []
    for t, h in zip(tracked, hist):
        p = o.token_probs(int(t))
        pvals.append(_chi2_pvalue(h, p, reps, chi2))
    np.savez_compressed(os.path.join(out, "ref_dist.npz"), params=json.dumps(REF_DIST), K=K, reps=reps,
                        tracked=tracked, hist=hist)
    pvals = np.array(pvals)
    return {"log": log.strip(), "tracked": len(tracked), "min_p": float(pvals.min()),
            "frac_p_below_0.01": float((pvals < 0.01).mean())}


def ezlda_timing(tmp, n=30, corpus=None):
    """EZLDA's per-sweep time (its own iterStart/iterStop events over its two-stream
    schedule, host<->device chunk copies included; EZLDA/mainKernel.cu:344-347,376) against
    this library on the same corpus and sweeps: resident (lda_trainer_iterate, CUDA events)
    and through host buffers (lda_iterate_host_async, topics uploaded and downloaded chunk
    by chunk every sweep, wall clock).  Both start from the corpus' initial topics; the LL
    of both final states is scored by the oracle's FP64 formula."""
    import time as _time
    import torch
    c = corpus if corpus is not None else make_corpus(REF_TIME)
    i = c.info
    d = os.path.join(tmp, "time")
    c.write_ezlda(d, K)
    dump = os.path.join(tmp, "time_out")
    os.makedirs(dump)
    t_ref = _time.perf_counter()
    log = run_harness("time", d, dump, n)
    t_ref = _time.perf_counter() - t_ref
    ref_ms = np.fromfile(os.path.join(dump, "sweep_ms.f32"), dtype=np.float32)
    z_ref = np.fromfile(os.path.join(dump, "topics_last.u16"), dtype=np.uint16) - 1
    tr = L.Trainer(c, K=K, alpha=float(ALPHA), beta=float(BETA), seed=42)
    stream = torch.cuda.current_stream()
    tr.set_stream(stream.cuda_stream)
    z0 = c.topics()
    tr.iterate(2)
    tr.set_topics(z0)
    tr.iteration = 0
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    tr.iterate(n)
    e1.record(stream)
    torch.cuda.synchronize()
    ours_ms = e0.elapsed_time(e1) / n
    z_ours = tr.topics()
    a = torch.from_numpy(z0.view(np.int16).copy()).pin_memory()
    b = torch.empty_like(a).pin_memory()
    tr.set_topics(z0)
    tr.iteration = 0
    torch.cuda.synchronize()
    t0 = _time.perf_counter()
    for _ in range(n):
        tr.iterate_host_async(a.numpy().view(np.uint16), b.numpy().view(np.uint16))
        a, b = b, a
    tr.wait()
    e2e_ms = 1e3 * (_time.perf_counter() - t0) / n
    same = bool(np.array_equal(a.numpy().view(np.uint16), z_ours))
    tr.close()
    o = Oracle(c.tok_word(), c.tok_doc(), i.vocab, i.num_docs, K, ALPHA, BETA)
    ll_ref, ll_ours = oracle_ll(o, z_ref.astype(np.uint16)), oracle_ll(o, z_ours)
    o.close()
    return {"log": log.strip(), "tokens": i.num_tokens, "sweeps": n, "harness_wall_s": t_ref,
            "ref_ms_per_sweep": float(ref_ms.mean()), "ref_ms_first_last": [float(ref_ms[0]), float(ref_ms[-1])],
            "ours_ms_per_sweep": ours_ms, "ours_e2e_ms_per_sweep": e2e_ms,
            "speedup_resident": float(ref_ms.mean()) / ours_ms, "speedup_e2e": float(ref_ms.mean()) / e2e_ms,
            "host_sweeps_equal_resident": same,
            "ll_after": {"ref": ll_ref, "ours": ll_ours, "rel_diff": abs(ll_ours - ll_ref) / abs(ll_ref)}}


def mode_time(tmp, out, n=30):
    res = ezlda_timing(tmp, n)
    with open(os.path.join(out, "ref_time.json"), "w") as f:
        json.dump({"params": REF_TIME, **res}, f, indent=1)
    return res


def _chi2_pvalue(h, p, n, chi2):
    """Pearson chi-square with bins of expected count < 5 pooled into one."""
    exp = p * n
    big = exp >= 5
    obs = list(h[big]) + [h[~big].sum()]
    ex = list(exp[big]) + [exp[~big].sum()]
    obs, ex = np.array(obs, float), np.array(ex, float)
    keep = ex > 0
    stat = (((obs - ex) ** 2)[keep] / ex[keep]).sum()
    dof = max(int(keep.sum()) - 1, 1)
    return float(chi2.sf(stat, dof))


def main():
    out = sys.argv[1] if len(sys.argv) > 1 else "ref_out"
    modes = "counts,sweeps,dist"
    sweeps = 100
    for a in sys.argv[2:]:
        if a.startswith("--modes="):
            modes = a.split("=", 1)[1]
        elif a.startswith("--sweeps="):
            sweeps = int(a.split("=", 1)[1])
    os.makedirs(out, exist_ok=True)
    tmp = tempfile.mkdtemp(prefix="ezlda_ref_")
    summary = {}
    try:
        for m in modes.split(","):
            fn = {"counts": mode_counts, "sweeps": lambda t, o: mode_sweeps(t, o, sweeps), "dist": mode_dist,
                  "time": mode_time}[m]
            try:
                summary[m] = fn(tmp, out)
            except Exception as e:  # record and continue with the other modes
                summary[m] = {"error": repr(e)}
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    with open(os.path.join(out, "summary.json"), "w") as f:
        json.dump(summary, f, indent=1)
    print(json.dumps(summary, indent=1))


if __name__ == "__main__":
    main()
