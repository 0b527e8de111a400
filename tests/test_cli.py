"""The ezlda_compat command-line driver (EZLDA/mainKernel.cu's surface) on a chunk directory."""
import os
import re
import subprocess

import numpy as np
import pytest

import lda_sc20_b200 as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "lda_sc20_b200", "ezlda_compat")


def test_cli_usage_and_bad_directory(tmp_path):
    r = subprocess.run([CLI, "--help"], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr
    r = subprocess.run([CLI, str(tmp_path / "none")], capture_output=True, text=True)
    assert r.returncode == 1 and "lengthVec.txt" in r.stderr


@pytest.mark.gpu
def test_cli_runs_sweeps_and_prints_ll(tmp_path):
    c = L.Corpus.generate(L.corpus_config("c0", num_chunks=2))
    d = str(tmp_path / "chunks")
    c.write_ezlda(d, 64)
    rec = str(tmp_path / "SamplingDRecord.txt")
    ck = str(tmp_path / "ck.bin")
    r = subprocess.run([CLI, d, "--K", "64", "--iters", "3", "--record", rec, "--checkpoint", ck],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lls = [float(x) for x in re.findall(r"^iter \d+ loglik (\S+)", r.stdout, re.M)]
    avg = [float(x) for x in re.findall(r"^Average Perplexity:(\S+)", r.stdout, re.M)]
    assert len(lls) == 3 and len(avg) == 3
    assert len(open(rec).read().split()) == 3
    # the same sweeps through the library from the loaded directory
    t = L.Trainer(L.Corpus.load_ezlda(d), K=64)
    for want in lls:
        got = t.iterate(1, ll=True)
        assert abs(got - want) <= 1e-6 * abs(want)
    t2 = L.Trainer(L.Corpus.load_ezlda(d), K=64)
    t2.restore(ck)
    assert t2.iteration == 3 and np.array_equal(t2.topics(), t.topics())


@pytest.mark.gpu
def test_cli_streams_chunks(tmp_path):
    """--streams streams the chunks (EZLDA's mode of operation) with the same LL line."""
    c = L.Corpus.generate(L.corpus_config("c0", num_chunks=3))
    d = str(tmp_path / "chunks")
    c.write_ezlda(d, 64)
    out = []
    for extra in ([], ["--streams", "2"]):
        r = subprocess.run([CLI, d, "--K", "64", "--iters", "2", "--record", ""] + extra,
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        out.append([float(x) for x in re.findall(r"^iter \d+ loglik (\S+)", r.stdout, re.M)])
        if extra:
            assert "chunks streamed through 2 CUDA streams" in r.stdout
    assert out[0] == out[1]

