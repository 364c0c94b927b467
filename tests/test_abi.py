"""The C ABI library, without a GPU: it builds for sm_100a, loads, exports
every entry point include/tsetlin_b200.h declares, and its host-side
argument checks answer the way the reference's do (capi.c:463-472,
1487, 1593, 757-775) before any device work."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "tsetlin_b200.h")
CSRC = os.path.join(ROOT, "lua-santoku-tsetlin_b200", "csrc")
LIB = os.path.join(ROOT, "lua-santoku-tsetlin_b200", "libtsetlin_b200.so")


@pytest.fixture(scope="module")
def so():
    if not os.path.exists(LIB):
        subprocess.run(["make", "-s", "-C", CSRC], check=True)
    return ctypes.CDLL(LIB)


def declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"\b(tm_[a-z_0-9]+)\s*\(", txt)))


def test_exports_every_declared_symbol(so):
    names = declared()
    assert "tm_create" in names and "tm_train" in names and "tm_predict" in names
    missing = [n for n in names if not hasattr(so, n)]
    assert not missing, missing


def test_python_mirror_lists_every_declared_symbol():
    import santoku_tsetlin as tm
    assert set(declared()) == set(tm.EXPORTS)


def test_python_mirror_types_every_argument():
    """Every entry point that takes arguments has its ctypes argument types
    set in the mirror (an untyped pointer argument would be converted as a
    C int), with as many types as the header declares parameters."""
    import santoku_tsetlin as tm
    txt = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    L = tm.lib()
    for name in declared():
        m = re.search(r"\b%s\s*\(([^)]*)\)" % name, txt)
        params = m.group(1).strip()
        n = 0 if params in ("", "void") else params.count(",") + 1
        f = getattr(L, name)
        if n == 0:
            assert not f.argtypes, name
        else:
            assert f.argtypes is not None and len(f.argtypes) == n, (name, n, f.argtypes)


def test_align_and_errors_without_gpu(so):
    import santoku_tsetlin as tm
    assert tm.lib().tm_align() == 8 == tm.align
    bad = [
        ({"classes": 0}, "classes"),
        ({"clauses": 0}, "clauses"),
        ({"clause_tolerance": 0}, "clause_tolerance"),
        ({"clause_maximum": 0}, "clause_maximum"),
        ({"state": 1}, "bits"),
    ]
    base = dict(classes=2, features=8, clauses=8, clause_tolerance=4, clause_maximum=4,
                specificity=2.0)
    for override, word in bad:
        t = dict(base, **override)
        with pytest.raises(tm.TsetlinError, match=word):
            tm.create("classifier", t)
    with pytest.raises(tm.TsetlinError, match="unexpected tsetlin machine type"):
        tm.create("regressor", base)
    with pytest.raises(tm.TsetlinError, match="feat_offsets"):
        tm.create("encoder", dict(hidden=3, clauses=8, clause_tolerance=4, clause_maximum=4,
                                  specificity=2.0, individualized=True,
                                  feat_offsets=np.array([0, 1, 2])))


def test_load_rejects_bad_data(so):
    import santoku_tsetlin as tm
    with pytest.raises(tm.TsetlinError, match="unexpected tsetlin machine type"):
        tm.load(np.array([7, 0, 0, 0], dtype=np.uint8).tobytes(), True)
    with pytest.raises(tm.TsetlinError, match="truncated"):
        tm.load(np.array([0, 0, 0, 0, 1, 0], dtype=np.uint8).tobytes(), True)
    with pytest.raises(tm.TsetlinError, match="cannot open"):
        tm.load("/nonexistent/model.bin")


def test_package_fails_loudly_without_the_library(tmp_path):
    """The package has no CPU fallback: without the built CUDA library every
    call raises instead of computing something another way."""
    import subprocess
    import sys
    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "import santoku_tsetlin as tm\n"
        "tm.LIB_PATH = %r\n"
        "try:\n"
        "    tm.create('classifier', dict(classes=2, features=8, clauses=8,\n"
        "              clause_tolerance=4, clause_maximum=4, specificity=2.0))\n"
        "except tm.TsetlinError as e:\n"
        "    print('RAISED', e)\n"
    ) % (os.path.join(ROOT, "lua-santoku-tsetlin_b200"), str(tmp_path / "missing.so"))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "RAISED" in r.stdout and "not built" in r.stdout
