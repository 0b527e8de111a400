"""The CUDA trainer's log-likelihood curve against the reference's own.

tests/golden/ref_ll.json holds the per-token log-likelihood of EZLDA's sampler
(LDAKernelTrain, EZLDA/utility.cu:1217-1611, driven in EZLDA/mainKernel.cu order by
oracle/ref/ref_harness) after each of 100 sweeps at K=1024 (EZLDA/mainKernel.cu:51
numIters = 100) from the corpus' initial topics, scored with the FP64 form of
profilePerp/utility.cu:2398,2810.  The CUDA trainer starts from the same topics and must
stay within 0.5% of that curve at every sweep.  The two chains use different random
streams (curand XORWOW against counter-based Philox), so they agree in distribution, not
token for token."""
import json
import os

import pytest

import lda_sc20_b200 as L

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
LL_REL_TOL = 5e-3  # 0.5% at every sweep


def test_ll_curve_within_half_percent_of_reference_over_100_sweeps():
    with open(os.path.join(HERE, "golden", "ref_ll.json")) as f:
        d = json.load(f)
    ref = d["ll_per_token_after_sweep"]
    assert len(ref) >= 101, "the fixture must cover 100 reference sweeps"
    p = dict(d["params"])
    c = L.Corpus.generate(L.corpus_config(p.pop("preset"), **p))
    assert c.info.num_tokens == d["tokens"]
    tr = L.Trainer(c, K=d["K"], alpha=d["alpha"], beta=d["beta"], seed=42)
    worst = 0.0
    for s, r in enumerate(ref):
        # an LL-mode sweep reports the likelihood of the topics it starts from: after s sweeps
        ll = tr.iterate(1, ll=True)
        rel = abs(ll - r) / abs(r)
        worst = max(worst, rel)
        assert rel <= LL_REL_TOL, f"after {s} sweeps: ours {ll:.6f} reference {r:.6f} ({100 * rel:.3f}%)"
    # the chain has moved well beyond the initial state, so the agreement is not trivial
    assert ref[-1] - ref[0] > 0.3
    print(f"max relative LL difference over {len(ref) - 1} sweeps: {worst:.2e}")
