"""Continuous-batching predict server (tm_serve_*).

Requests of many sizes for several resident machines are submitted from
several threads while earlier ones are on the GPU; each result must equal
what tm_predict returns for that request alone (predict is integer
arithmetic: zero tolerance).  Also: the HBM budget decides how many launch
slots exist and refuses a budget that covers none; a request larger than a
slot is refused.
"""
import ctypes
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _machine(tm, kind, features, classes, clauses, seed):
    from santoku_tsetlin import datagen
    rng = np.random.default_rng(seed)
    n = 300
    x = datagen.flip_pack(rng.random((n, features)) < 0.2)
    if kind == "classifier":
        t = tm.create("classifier", dict(classes=classes, features=features, clauses=clauses,
                                         clause_tolerance=16, clause_maximum=32,
                                         specificity=6.0, seed=seed))
        t.train({"samples": n, "problems": x.ravel(),
                 "solutions": rng.integers(0, classes, size=n).astype(np.int64),
                 "iterations": 2})
    else:
        t = tm.create("encoder", dict(hidden=classes, visible=features, clauses=clauses,
                                      clause_tolerance=16, clause_maximum=32, specificity=6.0,
                                      seed=seed))
        t.train({"samples": n, "sentences": x.ravel(),
                 "codes": datagen.pack_bits(rng.random((n, classes)) < 0.5).ravel(),
                 "iterations": 2})
    return t


def _open(tm, machines, budget, inflight=4, batch=4096, queued=0):
    L = tm.lib()
    cfg = tm._ServerConfig(budget, inflight, batch, 0, 0, queued)
    hs = (ctypes.c_void_p * len(machines))(*[m.handle.value for m in machines])
    srv = ctypes.c_void_p()
    rc = L.tm_serve_open(ctypes.byref(cfg), hs, len(machines), ctypes.byref(srv))
    return rc, srv


def test_alone_equals_mixed(tm):
    L = tm.lib()
    ms = [_machine(tm, "classifier", 784, 10, 64, 1),
          _machine(tm, "encoder", 500, 20, 32, 2),
          _machine(tm, "classifier", 4096, 6, 24, 3)]
    infos = [m.info() for m in ms]
    rc, srv = _open(tm, ms, budget=1 << 30)
    assert rc == 0, L.tm_last_error()
    rng = np.random.default_rng(5)
    reqs = []
    for i in range(120):
        k = int(rng.integers(0, len(ms)))
        n = int(np.exp(rng.uniform(0, np.log(2048))))
        feats = infos[k]["features"]
        x = np.packbits(np.concatenate([(b := rng.random((n, feats)) < 0.2), ~b], axis=1),
                        axis=1, bitorder="little").ravel()
        reqs.append((k, n, x))
    ids = [None] * len(reqs)

    def submit(lo, hi):
        for i in range(lo, hi):
            k, n, x = reqs[i]
            rid = ctypes.c_uint64()
            assert L.tm_serve_submit(srv, k, x.ctypes.data, n, ctypes.byref(rid)) == 0
            ids[i] = rid.value

    th = [threading.Thread(target=submit, args=(j * 30, (j + 1) * 30)) for j in range(4)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    lat = []
    for i, (k, n, x) in enumerate(reqs):
        info = infos[k]
        if info["type"] == 0:
            out = np.zeros(n, dtype=np.int64)
            done = L.tm_serve_poll(srv, ids[i], out.ctypes.data, None, 30_000_000)
        else:
            out = np.zeros(n * info["class_chunks"], dtype=np.uint8)
            done = L.tm_serve_poll(srv, ids[i], None, out.ctypes.data, 30_000_000)
        assert done == 1, L.tm_last_error()
        assert np.array_equal(out, ms[k].predict(x, n)), "request %d differs from predict alone" % i
        us = ctypes.c_double()
        assert L.tm_serve_latency_us(srv, ids[i], ctypes.byref(us)) == 0
        lat.append(us.value)
        # the three phases (queue wait, host launch calls, device work and
        # completion) are non-negative and add up to the latency; the
        # launch's device span is positive
        ph = (ctypes.c_double * 4)()
        assert L.tm_serve_phases_us(srv, ids[i], ph) == 0
        assert min(ph[:3]) >= 0 and abs(sum(ph[:3]) - us.value) <= 1e-6 * us.value + 1e-3
        assert ph[3] > 0
    assert all(v > 0 for v in lat)
    # a polled request is released: its id is unknown to a second poll, its
    # latency stays readable, and nothing is left waiting
    out = np.zeros(4096, dtype=np.int64)
    assert L.tm_serve_poll(srv, ids[0], out.ctypes.data, out.ctypes.data, 0) < 0
    assert b"unknown" in L.tm_last_error()
    st = np.zeros(5, dtype=np.uint64)
    assert L.tm_serve_stats(srv, st.ctypes.data) == 0
    assert st[0] == 0 and st[1] == 0 and st[2] == 0 and st[3] == 0 and st[4] >= 1
    assert L.tm_serve_close(srv) == 0


def test_budget_and_oversized_requests(tm):
    L = tm.lib()
    m = _machine(tm, "classifier", 784, 10, 16, 4)
    rc, _ = _open(tm, [m], budget=1024)
    assert rc < 0 and b"budget" in L.tm_last_error()
    rc, srv = _open(tm, [m], budget=1 << 28, inflight=2, batch=64)
    assert rc == 0
    x = np.zeros(65 * 196, dtype=np.uint8)
    rid = ctypes.c_uint64()
    assert L.tm_serve_submit(srv, 0, x.ctypes.data, 65, ctypes.byref(rid)) < 0
    assert L.tm_serve_submit(srv, 0, x.ctypes.data, 64, ctypes.byref(rid)) == 0
    out = np.zeros(64, dtype=np.int64)
    assert L.tm_serve_poll(srv, rid.value, out.ctypes.data, None, 10_000_000) == 1
    assert np.array_equal(out, m.predict(x, 64))
    assert L.tm_serve_close(srv) == 0


def test_queue_bound_refuses_with_busy(tm):
    """A full queue refuses new requests with TM_ERR_BUSY (-7) instead of
    letting the backlog grow without bound; refused requests can be
    submitted again once the queue drains, and accepted ones complete
    exactly."""
    L = tm.lib()
    m = _machine(tm, "classifier", 4096, 6, 64, 7)
    # one slot of 256 samples, at most 512 samples waiting
    rc, srv = _open(tm, [m], budget=1 << 30, inflight=1, batch=256, queued=512)
    assert rc == 0, L.tm_last_error()
    rng = np.random.default_rng(3)
    x = np.packbits(np.concatenate([(b := rng.random((256, 4096)) < 0.2), ~b], axis=1), axis=1,
                    bitorder="little").ravel()
    want = m.predict(x, 256)
    ok, busy = [], 0
    for _ in range(40):
        rid = ctypes.c_uint64()
        rc = L.tm_serve_submit(srv, 0, x.ctypes.data, 256, ctypes.byref(rid))
        if rc == 0:
            ok.append(rid.value)
        else:
            assert rc == -7 and b"queue full" in L.tm_last_error()
            busy += 1
    assert busy > 0 and len(ok) >= 2
    for rid in ok:
        out = np.zeros(256, dtype=np.int64)
        assert L.tm_serve_poll(srv, rid, out.ctypes.data, None, 30_000_000) == 1
        assert np.array_equal(out, want)
    rid = ctypes.c_uint64()
    assert L.tm_serve_submit(srv, 0, x.ctypes.data, 256, ctypes.byref(rid)) == 0
    out = np.zeros(256, dtype=np.int64)
    assert L.tm_serve_poll(srv, rid.value, out.ctypes.data, None, 30_000_000) == 1
    assert np.array_equal(out, want)
    assert L.tm_serve_close(srv) == 0


def test_small_requests_of_many_machines_share_launches(tm):
    """Requests of 1-40 samples for different machines -- packed into the
    same launch slots, the small ones as warp-per-clause jobs -- each equal
    tm_predict alone."""
    L = tm.lib()
    ms = [_machine(tm, "classifier", 16384, 5, 24, 11), _machine(tm, "encoder", 700, 13, 16, 12),
          _machine(tm, "classifier", 784, 10, 40, 13)]
    infos = [m.info() for m in ms]
    rc, srv = _open(tm, ms, budget=1 << 30, inflight=2, batch=512)
    assert rc == 0, L.tm_last_error()
    rng = np.random.default_rng(9)
    reqs = []
    for i in range(90):
        k = i % 3
        n = int(rng.integers(1, 41))
        feats = infos[k]["features"]
        x = np.packbits(np.concatenate([(b := rng.random((n, feats)) < 0.1), ~b], axis=1),
                        axis=1, bitorder="little").ravel()
        rid = ctypes.c_uint64()
        assert L.tm_serve_submit(srv, k, x.ctypes.data, n, ctypes.byref(rid)) == 0
        reqs.append((k, n, x, rid.value))
    for k, n, x, rid in reqs:
        info = infos[k]
        out = np.zeros(n * (8 if info["type"] == 0 else info["class_chunks"]), dtype=np.uint8)
        assert L.tm_serve_poll(srv, rid, out.ctypes.data, out.ctypes.data, 30_000_000) == 1
        got = out.view(np.int64) if info["type"] == 0 else out
        assert np.array_equal(got, ms[k].predict(x, n))
    assert L.tm_serve_close(srv) == 0


def test_large_requests_through_gemm_match_oracle(tm):
    """Requests large enough for the 8-bit GEMM path (packed with small
    ones in the same slots) give the oracle's bitwise predictions: a
    classifier on 1,024-word rows and an encoder on 256-word rows, random
    actions of clauses short enough that the votes depend on the exact
    failed-literal counts."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from test_gpu_gemm_predict import _machine_pair
    L = tm.lib()
    pairs = [_machine_pair(tm, "classifier", 20, 16384, 64, 0.0005, 21),
             _machine_pair(tm, "encoder", 24, 4096, 48, 0.004, 22)]
    ms = [t for _, t, _ in pairs]
    infos = [t.info() for t in ms]
    rc, srv = _open(tm, ms, budget=1 << 31, inflight=3, batch=2048)
    assert rc == 0, L.tm_last_error()
    rng = np.random.default_rng(23)
    reqs = []
    for n in (300, 2000, 7, 1000, 40, 1500, 1, 600):
        for k in range(2):
            feats = infos[k]["features"]
            b = rng.random((n, feats)) < 0.02
            x = np.packbits(np.concatenate([b, ~b], axis=1), axis=1, bitorder="little").ravel()
            rid = ctypes.c_uint64()
            assert L.tm_serve_submit(srv, k, x.ctypes.data, n, ctypes.byref(rid)) == 0
            reqs.append((k, n, x, rid.value))
    for k, n, x, rid in reqs:
        info = infos[k]
        out = np.zeros(n * (8 if info["type"] == 0 else info["class_chunks"]), dtype=np.uint8)
        assert L.tm_serve_poll(srv, rid, out.ctypes.data, out.ctypes.data, 60_000_000) == 1
        got = out.view(np.int64) if info["type"] == 0 else out
        want = np.asarray(pairs[k][0].predict(x, n)).ravel()
        if info["type"] == 0:
            assert np.array_equal(got, want), (k, n)
        else:
            # codes compared within the hidden bits of each sample's last byte
            nb = info["class_chunks"]
            mask = np.full(nb, 0xFF, dtype=np.uint8)
            if info["classes"] % 8:
                mask[-1] = (1 << (info["classes"] % 8)) - 1
            assert np.array_equal(got.reshape(n, nb) & mask,
                                  want.astype(np.uint8).reshape(n, nb) & mask), (k, n)
    assert L.tm_serve_close(srv) == 0
    for t in ms:
        t.destroy()
