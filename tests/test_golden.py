"""The oracle against golden fixtures produced by EZLDA's own kernels.

The fixtures in tests/golden/ were written by oracle/ref/run_ref.py, which runs the
reference's unmodified EZLDA/*.cu (built into oracle/_ref by oracle/ref/build_ref.py) on
seeded corpora.  The corpora are regenerated here from the parameters stored with each
fixture."""
import json
import os

import numpy as np
import pytest

import lda_sc20_b200 as L
from oracle import Oracle

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def _fixture(name):
    p = os.path.join(GOLDEN, name)
    if not os.path.exists(p):
        pytest.skip(f"{name} not generated")
    return p


def _corpus(params):
    p = dict(params)
    preset = p.pop("preset")
    return L.Corpus.generate(L.corpus_config(preset, **p))


def test_counts_match_reference_kernels():
    """n_k, sparse and dense word-topic counts, DT rows and per-token doc metadata equal
    EZLDA's rebuild kernels bit for bit; max/2nd/3rd topics equal EZLDA's except where
    phi ties; Q equals EZLDA's sum(phi) - phi_max to float rounding."""
    from oracle.ref.run_ref import compare_counts
    z = np.load(_fixture("ref_counts.npz"))
    params = json.loads(str(z["params"]))
    ref = {k: z[k] for k in z.files if k not in ("params", "K")}
    c = _corpus(params)
    res = compare_counts(c, ref)
    for key in ("n_k", "dense_wt", "sparse_wt", "doc_rows", "doc_ids", "token_meta", "max_topic_ties_only"):
        assert res[key], (key, res)
    assert res["q_max_rel_diff"] < 1e-5
    # words that never occur have a constant phi column (ties everywhere); every
    # disagreement is an exact tie (checked above), and most words agree outright
    same = res["max_topic_same"]
    assert same[0] >= 0.95 * same[3]


def test_reference_sampler_draws_from_the_oracle_conditional():
    """Draws of EZLDA's LDAKernelTrain over 2,000 independent sweeps from one state,
    chi-squared against the oracle's exact FP64 conditional p(k) ∝ (n_dk+α)(n_wk+β)/(n_k+Vβ)."""
    from scipy.stats import chi2
    from oracle.ref.run_ref import ALPHA, BETA, K, _chi2_pvalue
    z = np.load(_fixture("ref_dist.npz"))
    params = json.loads(str(z["params"]))
    reps = int(z["reps"])
    c = _corpus(params)
    i = c.info
    o = Oracle(c.tok_word(), c.tok_doc(), i.vocab, i.num_docs, K, ALPHA, BETA)
    o.rebuild(c.topics())
    pv = np.array([_chi2_pvalue(h, o.token_probs(int(t)), reps, chi2) for t, h in zip(z["tracked"], z["hist"])])
    assert len(pv) >= 50
    # under the null the p-values are uniform: few small ones, and Fisher's combination holds
    assert (pv < 1e-3).sum() <= 2
    stat = -2 * np.log(np.maximum(pv, 1e-300)).sum()
    assert chi2.sf(stat, 2 * len(pv)) > 1e-4


def test_oracle_ll_curve_tracks_reference():
    """The oracle's chain from the reference's initial topics follows the reference's
    per-sweep log-likelihood within 0.5% at every committed sweep (100 at K=1024)."""
    from oracle.ref.run_ref import ALPHA, BETA, K, oracle_ll
    d = json.load(open(_fixture("ref_ll.json")))
    ref = d["ll_per_token_after_sweep"]
    c = _corpus(d["params"])
    i = c.info
    assert i.num_tokens == d["tokens"]
    o = Oracle(c.tok_word(), c.tok_doc(), i.vocab, i.num_docs, K, ALPHA, BETA)
    zz = c.topics()
    # same state: only the float summation order of S inside the FP64 log can differ
    assert abs(oracle_ll(o, zz) - ref[0]) <= 1e-6 * abs(ref[0])
    for s in range(1, len(ref)):
        # an LL-mode sweep scores the state it starts from, i.e. after s - 1 sweeps
        st = o.iterate(zz, 42, s - 1, ll=True)
        ll = st.loglik / st.tokens
        assert abs(ll - ref[s - 1]) <= 5e-3 * abs(ref[s - 1]), (s - 1, ll, ref[s - 1])
    ll = oracle_ll(o, zz)
    assert abs(ll - ref[-1]) <= 5e-3 * abs(ref[-1]), (len(ref) - 1, ll, ref[-1])
