"""Edge cases of the machine's parameter space, CUDA path against the oracle
(bit-exact state, vote sums and outputs): the smallest machine (one class,
one feature, 2-bit automata), include_bits equal to state_bits, a tolerance
of 1 and one far above the literal count, an encoder whose hidden width is
not a multiple of 8 (the reference leaves the padding bits of the last code
byte stale, capi.c:957-990, so codes are compared within `hidden`), empty
predicts, and a predict larger than one tile row in every dimension."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from test_gpu_parity import _oracle_pair, ref_table, train_table  # noqa: E402

pytestmark = pytest.mark.gpu

EDGES = [
    dict(type="classifier", classes=1, features=1, clauses=8, clause_tolerance=1,
         clause_maximum=1, state=2, specificity=1.5, target=1),
    dict(type="classifier", classes=3, features=37, clauses=8, clause_tolerance=3,
         clause_maximum=5, state=3, include_bits=3, specificity=2.0, target=0.25),
    dict(type="classifier", classes=5, features=90, clauses=24, clause_tolerance=500,
         clause_maximum=500, state=8, include_bits=1, specificity=30.0, target=40),
    dict(type="encoder", classes=13, features=45, clauses=16, clause_tolerance=6,
         clause_maximum=12, state=5, include_bits=2, specificity=4.0, target=6),
    dict(type="encoder", classes=1, features=300, clauses=8, clause_tolerance=8,
         clause_maximum=40, state=8, specificity=10.0, target=-1),
]


def _inputs(cfg, n, nt, seed):
    from santoku_tsetlin import datagen
    rng = np.random.default_rng(seed)
    x = datagen.flip_pack(rng.random((n + nt, cfg["features"])) < 0.3)
    inp = dict(n=n, x=x[:n].ravel())
    if cfg["type"] == "classifier":
        inp["labels"] = rng.integers(0, cfg["classes"], size=n).astype(np.int64)
    else:
        nb = (cfg["classes"] + 7) // 8
        inp["codes"] = rng.integers(0, 256, size=n * nb).astype(np.uint8)
    return inp, x[n:].ravel()


@pytest.mark.parametrize("cfg", EDGES, ids=["smallest", "ib_eq_state", "tol_above_literals",
                                            "enc_hidden13", "enc_hidden1"])
def test_edge_machines_match_oracle(tm, cfg):
    n, nt = 120, 70
    inp, xt = _inputs(cfg, n, nt, seed=len(str(cfg)))
    m = _oracle_pair(cfg["type"], cfg, inp, 3, seed=9)
    kind, tbl = ref_table(cfg, seed=9)
    t = tm.create(kind, tbl)
    t.train(train_table(kind, inp, 3))
    a, s = t.export_state()
    assert np.array_equal(a, m.actions())
    assert np.array_equal(s, m.state())
    assert np.array_equal(t.predict_scores(xt, nt), m.predict(xt, nt, scores=True)[1])
    got = np.asarray(t.predict(xt, nt))
    want = m.predict(xt, nt)
    if kind == "encoder":
        # compare code bits within `hidden` (the reference leaves padding bits stale)
        nb = (cfg["classes"] + 7) // 8
        bits = lambda v: np.unpackbits(np.asarray(v, np.uint8).reshape(nt, nb), axis=1,
                                       bitorder="little", count=cfg["classes"])
        assert np.array_equal(bits(got), bits(want))
    else:
        assert np.array_equal(got, np.asarray(want))
    # an empty predict returns an empty result
    assert np.asarray(t.predict(xt[:0], 0)).size == 0
    t.destroy()


def test_predict_spans_many_tiles(tm):
    """More samples, clauses and words than one 64 x 64 x 32 tile: vote sums
    equal the oracle's on a machine with random actions."""
    cfg = dict(type="classifier", classes=3, features=1500, clauses=200, clause_tolerance=40,
               clause_maximum=200, specificity=10.0, target=30)
    rng = np.random.default_rng(77)
    kind, tbl = ref_table(cfg, seed=1)
    t = tm.create(kind, tbl)
    info = t.info()
    acts = (rng.random(info["action_chunks"]) < 0.01).astype(np.uint8) * rng.integers(
        0, 256, size=info["action_chunks"]).astype(np.uint8)
    t.import_state(acts, None)
    import oracle as O
    m = O.Machine(**cfg)
    m.load_state(acts, None)
    nt = 1000
    xt = np.packbits(rng.random((nt, 3000)) < 0.5, axis=1, bitorder="little").ravel()
    assert np.array_equal(t.predict_scores(xt, nt), m.predict(xt, nt, scores=True)[1])
    assert np.array_equal(np.asarray(t.predict(xt, nt)), np.asarray(m.predict(xt, nt)))
    t.destroy()
