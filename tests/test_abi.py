"""CPU tests of the C ABI boundary: the library loads, exports every declared entry point,
and reports host-side errors as status codes (no compute without a GPU)."""
import ctypes
import os
import re

import pytest

import lda_sc20_b200 as L
from lda_sc20_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    names = []
    for hdr in os.listdir(os.path.join(ROOT, "include")):
        if not hdr.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", hdr)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(lda_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = _native.load()
    names = _declared_functions()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    names = set(_declared_functions())
    assert names <= set(_native.SIGNATURES), sorted(names - set(_native.SIGNATURES))


def test_version_and_error_text():
    lib = _native.load()
    assert b"sm_100a" in lib.lda_version()
    with pytest.raises(L.LdaError) as e:
        L.Corpus.load_ezlda("/nonexistent/dir")
    assert "lengthVec.txt" in str(e.value)


def test_null_arguments_are_rejected():
    lib = _native.load()
    assert lib.lda_corpus_generate(None, None) == -1
    assert lib.lda_trainer_iterate(None, 1, 0) == -1
    assert lib.lda_update_wt(None) == -1
    assert lib.lda_trainer_create(None, None, None) == -1


def test_trainer_config_validation_is_host_side():
    c = L.Corpus.generate(L.corpus_config("c0"))
    with pytest.raises(L.LdaError) as e:
        L.Trainer(c, K=3)
    assert e.value.code == -1
    with pytest.raises(L.LdaError) as e:
        L.Trainer(c, K=32)  # initial topics drawn for K=64
    assert e.value.code == -1
