"""Randomized parity sweep: seeded random machines across the parameter space
(classifier / encoder, dense / individualized, 2-12 state bits, include
bits 1-3, feature counts with and without tail masks, tolerance, maximum,
target given, fractional or default, specificity) trained for two epochs on
random data; the CUDA path's automaton state, vote sums and outputs equal
the oracle's bit for bit.  The automatic variant choice picks whichever
train kernel is fastest for each shape, so the sweep also crosses variants."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from test_gpu_parity import _oracle_pair, ref_table, train_table  # noqa: E402

pytestmark = pytest.mark.gpu


def _random_case(seed):
    r = np.random.default_rng(1000 + seed)
    kind = "encoder" if r.random() < 0.4 else "classifier"
    ind = r.random() < 0.3
    classes = int(r.integers(1, 12))
    state = int(r.choice([2, 3, 5, 8, 8, 8, 10, 12]))
    cfg = dict(type=kind, classes=classes, clauses=int(8 * r.integers(1, 7)),
               clause_tolerance=int(r.integers(1, 60)), clause_maximum=int(r.integers(1, 200)),
               state=state, include_bits=int(r.integers(1, min(3, state) + 1)),
               specificity=float(r.uniform(1.5, 30.0)))
    t = r.random()
    cfg["target"] = -1.0 if t < 0.25 else (float(r.uniform(0.05, 0.9)) if t < 0.5
                                           else int(r.integers(1, 80)))
    n, nt = int(r.integers(20, 150)), int(r.integers(1, 60))
    inp = dict(n=n)
    if ind:
        cfg["individualized"] = True
        ks = r.integers(1, 140, size=classes)
        fo = np.concatenate([[0], np.cumsum(ks)]).astype(np.int64)
        cfg["feat_offsets"] = fo
        from santoku_tsetlin import datagen

        def pack(nn):
            blocks, offs, off = [], [], 0
            for h in range(classes):
                xb = datagen.flip_pack(r.random((nn, ks[h])) < r.uniform(0.05, 0.5)).ravel()
                offs.append(off)
                off += xb.size
                blocks.append(xb)
            return np.concatenate(blocks), np.array(offs, dtype=np.int64)
        inp["x"], inp["dim_offsets"] = pack(n)
        xt, doff_t = pack(nt)
    else:
        from santoku_tsetlin import datagen
        F = int(r.integers(1, 700))
        cfg["features"] = F
        x = datagen.flip_pack(r.random((n + nt, F)) < r.uniform(0.05, 0.5))
        inp["x"] = x[:n].ravel()
        xt, doff_t = x[n:].ravel(), None
    if kind == "classifier":
        inp["labels"] = r.integers(0, classes + (1 if r.random() < 0.2 else 0), size=n).astype(np.int64)
    else:
        inp["codes"] = r.integers(0, 256, size=n * ((classes + 7) // 8)).astype(np.uint8)
    return cfg, inp, xt, doff_t, nt


@pytest.mark.parametrize("seed", range(16))
def test_random_machine_matches_oracle(tm, seed):
    cfg, inp, xt, doff_t, nt = _random_case(seed)
    m = _oracle_pair(cfg["type"], cfg, inp, 2, seed=seed)
    kind, tbl = ref_table(cfg, seed=seed)
    t = tm.create(kind, tbl)
    t.train(train_table(kind, inp, 2))
    a, s = t.export_state()
    assert np.array_equal(a, m.actions()), cfg
    assert np.array_equal(s, m.state()), cfg
    pargs = (xt, doff_t, nt) if doff_t is not None else (xt, nt)
    want_out, want_scores = m.predict(xt, nt, dim_offsets=doff_t, scores=True)
    assert np.array_equal(t.predict_scores(*pargs), want_scores), cfg
    got = np.asarray(t.predict(*pargs))
    if kind == "encoder":
        nb = (cfg["classes"] + 7) // 8
        bits = lambda v: np.unpackbits(np.asarray(v, np.uint8).reshape(nt, nb), axis=1,
                                       bitorder="little", count=cfg["classes"])
        assert np.array_equal(bits(got), bits(want_out)), cfg
    else:
        assert np.array_equal(got, np.asarray(want_out)), cfg
    t.destroy()
