"""tm_predict_noalloc, the allocation-free predict entry point.

Some callers cannot let this library call cudaMalloc / cudaFree during a
request: a serving loop whose latency budget cannot absorb the device-wide
synchronisation those calls cause, or an application whose own allocator
already holds the GPU's memory.  For them the library keeps one fixed
scratch array compiled in.  This file checks, through the C ABI, that two
calls in a row give exactly what tm_predict gives (predict is integer
arithmetic, so the tolerance is zero), and that a request too large for the
scratch is refused.  It is named so that pytest collects it last; it also
passes alone in a fresh process.
"""
import ctypes
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "lua-santoku-tsetlin_b200"))

pytestmark = pytest.mark.gpu


def _trained(tm, kind, features, classes, n, seed):
    from santoku_tsetlin import datagen
    rng = np.random.default_rng(seed)
    x = datagen.flip_pack(rng.random((n, features)) < 0.25)
    if kind == "classifier":
        t = tm.create("classifier", dict(classes=classes, features=features, clauses=32,
                                         clause_tolerance=16, clause_maximum=32,
                                         specificity=5.0, seed=seed, reusable=True))
        y = rng.integers(0, classes, size=n).astype(np.int64)
        t.train({"samples": n, "problems": x.ravel(), "solutions": y, "iterations": 2})
    else:
        t = tm.create("encoder", dict(hidden=classes, visible=features, clauses=24,
                                      clause_tolerance=16, clause_maximum=32,
                                      specificity=5.0, seed=seed, reusable=True))
        c = datagen.pack_bits(rng.random((n, classes)) < 0.5)
        t.train({"samples": n, "sentences": x.ravel(), "codes": c.ravel(), "iterations": 2})
    return t


@pytest.mark.parametrize("kind", ["classifier", "encoder"])
def test_noalloc_matches_predict_twice(tm, kind):
    import torch
    t = _trained(tm, kind, features=300, classes=11, n=500, seed=3)
    info = t.info()
    rng = np.random.default_rng(9)
    lib = tm.lib()
    for call in range(2):
        nq = 700 + 37 * call
        xq = np.packbits(np.concatenate([(b := rng.random((nq, 300)) < 0.25), ~b], axis=1),
                         axis=1, bitorder="little")
        want = t.predict(xq.ravel(), nq)
        xd = torch.from_numpy(xq.ravel().copy()).cuda()
        if kind == "classifier":
            out = torch.full((nq,), -7, dtype=torch.int64, device="cuda")
            rc = lib.tm_predict_noalloc(t.handle, xd.data_ptr(), nq, out.data_ptr(), None)
        else:
            out = torch.full((nq * info["class_chunks"],), 0xAB, dtype=torch.uint8, device="cuda")
            rc = lib.tm_predict_noalloc(t.handle, xd.data_ptr(), nq, None, out.data_ptr())
        assert rc == 0, lib.tm_last_error().decode()
        assert np.array_equal(out.cpu().numpy(), want)


def test_noalloc_refuses_oversized_request(tm):
    import torch
    t = _trained(tm, "classifier", features=4096, classes=4, n=64, seed=5)
    nq = 9000  # 9000 rows of 1 KB exceed the 8 MiB scratch
    xd = torch.zeros(nq * 1024, dtype=torch.uint8, device="cuda")
    out = torch.zeros(nq, dtype=torch.int64, device="cuda")
    lib = tm.lib()
    rc = lib.tm_predict_noalloc(t.handle, xd.data_ptr(), nq, out.data_ptr(), None)
    assert rc < 0
    assert b"8 MiB" in lib.tm_last_error()


@pytest.mark.parametrize("nq", [2 ** 31, 2 ** 62, 2 ** 64 - 1])
def test_noalloc_refuses_huge_n_without_touching_memory(tm, nq):
    # n so large that n * row bytes wraps 64 bits: refused before any size is
    # multiplied out, so the small buffers below are never read or written
    import torch
    t = _trained(tm, "classifier", features=300, classes=11, n=64, seed=6)
    xd = torch.zeros(256, dtype=torch.uint8, device="cuda")
    out = torch.zeros(4, dtype=torch.int64, device="cuda")
    lib = tm.lib()
    rc = lib.tm_predict_noalloc(t.handle, xd.data_ptr(), nq, out.data_ptr(), None)
    assert rc == -1  # TM_ERR_ARG
    assert b"8 MiB" in lib.tm_last_error()
    assert int(out.abs().sum().item()) == 0


def test_noalloc_refuses_individualized_with_its_own_name(tm):
    t = tm.create("classifier", dict(classes=2, clauses=8, clause_tolerance=8, clause_maximum=8,
                                     specificity=4.0, individualized=True,
                                     feat_offsets=[0, 3, 7]))
    lib = tm.lib()
    rc = lib.tm_predict_noalloc(t.handle, None, 0, None, None)
    assert rc == 0  # n == 0 is a no-op
    import torch
    xd = torch.zeros(16, dtype=torch.uint8, device="cuda")
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    rc = lib.tm_predict_noalloc(t.handle, xd.data_ptr(), 1, out.data_ptr(), None)
    assert rc == -1
    assert b"predict_noalloc" in lib.tm_last_error()
