"""Parity of the CUDA path (through the C ABI) with the reference.

* Every golden fixture made from the reference's own capi.c/automata.h
  (tests/golden/make_golden.py): after training under the Philox draw
  contract the device automata, vote sums, predictions and persisted bytes
  are bit-identical.
* Larger machines against the CPU oracle (itself pinned to the fixtures).
* API behaviour of the reference: each-callback stop, persist/load,
  checkpoint/restore, reconfigure, restrict, device-pointer inputs.
"""
import hashlib
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from cases import CASES, make_inputs  # noqa: E402

import oracle as O  # noqa: E402

pytestmark = pytest.mark.gpu

PHILOX_CASES = [c for c in CASES if not c["train"].get("refstruct")]


def ref_table(create, seed=0, reusable=True):
    """Oracle-style create kwargs -> the reference's Lua table keys."""
    c = dict(create)
    kind = c.pop("type")
    t = {}
    if kind == "encoder":
        t["hidden"] = c.pop("classes")
        if "features" in c:
            t["visible"] = c.pop("features")
    for k, v in c.items():
        t[k] = v
    t["reusable"] = reusable
    t["seed"] = seed
    return kind, t


def train_table(kind, inp, epochs, seed=None):
    t = {"samples": inp["n"], "iterations": epochs}
    if kind == "classifier":
        t["problems"], t["solutions"] = inp["x"], inp["labels"]
    else:
        t["sentences"], t["codes"] = inp["x"], inp["codes"]
    if inp.get("dim_offsets") is not None:
        t["dim_offsets"] = inp["dim_offsets"]
    if seed is not None:
        t["seed"] = seed
    return t


def load_fixture(name):
    z = np.load(os.path.join(HERE, "golden", name + ".npz"))
    return {k: z[k] for k in z.files}


def predict_args(inp):
    if inp.get("dim_offsets_t") is not None:
        return (inp["xt"], inp["dim_offsets_t"], inp["nt"])
    return (inp["xt"], inp["nt"])


@pytest.mark.parametrize("variant", ["auto", "cta"])
@pytest.mark.parametrize("case", PHILOX_CASES, ids=[c["name"] for c in PHILOX_CASES])
def test_train_matches_reference_fixture(tm, monkeypatch, case, variant):
    # "auto": short rows train with one warp per unit; "cta": the one-CTA-per-
    # unit kernel on the same rows
    if variant == "cta":
        monkeypatch.setenv("TSETLIN_B200_NO_WARP", "1")
    case = dict(case, create=dict(case["create"]))
    inp = make_inputs(case)
    fx = load_fixture(case["name"])
    kind, tbl = ref_table(case["create"], seed=case["train"]["seed"])
    t = tm.create(kind, tbl)
    t.train(train_table(kind, inp, case["train"]["epochs"]))
    acts, state = t.export_state()
    assert np.array_equal(acts, fx["actions"]), "actions differ"
    assert hashlib.sha256(state.tobytes()).digest() == fx["state_sha256"].tobytes(), "state differs"
    scores = t.predict_scores(*predict_args(inp))
    assert np.array_equal(scores, fx["scores"])
    out = t.predict(*predict_args(inp))
    assert np.array_equal(out, fx["out"].ravel())
    assert t.persist() == fx["persist"].tobytes()
    info = dict(zip(fx["info_keys"].tolist(), fx["info_vals"].tolist()))
    got = t.info()
    for k in info:
        if k not in ("reusable", "has_state"):
            assert got[k] == info[k], k


def _oracle_pair(kind, create, inp, epochs, seed):
    m = O.Machine(**create)
    m.train(inp["x"], inp["n"], epochs, labels=inp.get("labels"), codes=inp.get("codes"),
            dim_offsets=inp.get("dim_offsets"), seed=seed)
    return m


@pytest.mark.parametrize("cfg", [
    dict(type="classifier", classes=10, features=784, clauses=64, clause_tolerance=64,
         clause_maximum=64, target=50, specificity=10.0, n=1500, epochs=3),
    dict(type="encoder", classes=16, features=300, clauses=32, clause_tolerance=16,
         clause_maximum=24, specificity=6.0, n=800, epochs=2),
    dict(type="classifier", classes=4, features=4500, clauses=16, clause_tolerance=32,
         clause_maximum=200, specificity=25.0, n=300, epochs=2),
], ids=["c0_like", "encoder", "wide_rows"])
def test_train_matches_oracle_larger(tm, cfg):
    from santoku_tsetlin import datagen
    cfg = dict(cfg)
    n, epochs = cfg.pop("n"), cfg.pop("epochs")
    rng = np.random.default_rng(5)
    kind = cfg["type"]
    if kind == "classifier" and cfg["features"] == 784:
        x, y, _ = datagen.prototype_classifier(n + 200, classes=cfg["classes"], seed=3)
        inp = dict(n=n, x=x[:n].ravel(), labels=y[:n], xt=x[n:].ravel(), nt=200)
    else:
        F = cfg["features"]
        x = datagen.flip_pack(rng.random((n + 100, F)) < 0.2)
        inp = dict(n=n, x=x[:n].ravel(), xt=x[n:].ravel(), nt=100)
        if kind == "classifier":
            inp["labels"] = rng.integers(0, cfg["classes"], size=n).astype(np.int64)
        else:
            inp["codes"] = datagen.pack_bits(rng.random((n, cfg["classes"])) < 0.5).ravel()
    m = _oracle_pair(kind, cfg, inp, epochs, seed=9)
    kind, tbl = ref_table(cfg, seed=9)
    t = tm.create(kind, tbl)
    t.train(train_table(kind, inp, epochs))
    a, s = t.export_state()
    assert np.array_equal(a, m.actions())
    assert np.array_equal(s, m.state())
    assert np.array_equal(t.predict_scores(inp["xt"], inp["nt"]),
                          m.predict(inp["xt"], inp["nt"], scores=True)[1])


def test_predict_random_actions_wide(tm):
    """Predict alone on wide rows and many clauses: random actions imported,
    vote sums and argmax against the oracle."""
    rng = np.random.default_rng(11)
    for kind, classes, F, clauses in (("classifier", 20, 16384, 64), ("encoder", 24, 4096, 40)):
        cfg = dict(type=kind, classes=classes, features=F, clauses=clauses, clause_tolerance=64,
                   clause_maximum=64, specificity=25.0)
        m = O.Machine(**cfg)
        nbytes = m.info["action_chunks"]
        acts = (rng.random(nbytes * 8) < 0.004)
        acts = np.packbits(acts, bitorder="little")
        m.load_state(actions=acts)
        n = 97
        x = np.packbits(np.concatenate([(b := rng.random((n, F)) < 0.02), ~b], axis=1), axis=1,
                        bitorder="little").ravel()
        kind2, tbl = ref_table(cfg)
        t = tm.create(kind2, tbl)
        t.import_state(actions=acts)
        want_out, want_sc = m.predict(x, n, scores=True)
        assert np.array_equal(t.predict_scores(x, n), want_sc)
        assert np.array_equal(t.predict(x, n), want_out.ravel())


def test_predict_ties_go_to_lowest_class(tm):
    t = tm.create("classifier", dict(classes=5, features=8, clauses=8, clause_tolerance=3,
                                     clause_maximum=3, specificity=2.0))
    # all actions zero: every clause is empty, fires with vote = tolerance,
    # even and odd cancel -> every class sums to 0 -> argmax is class 0
    x = np.zeros((10, 2), dtype=np.uint8)
    assert np.all(t.predict(x, 10) == 0)
    assert np.all(t.predict_scores(x, 10) == 0)


def test_each_callback_stops_training(tm):
    case = dict(CASES[0], create=dict(CASES[0]["create"]))
    inp = make_inputs(case)
    kind, tbl = ref_table(case["create"], seed=4)
    seen = []

    def each(epoch):
        seen.append(epoch)
        return epoch < 2

    t = tm.create(kind, tbl)
    t.train(dict(train_table(kind, inp, 5), each=each))
    assert seen == [1, 2]
    t2 = tm.create(kind, tbl)
    t2.train(train_table(kind, inp, 2))
    assert np.array_equal(t.export_state()[0], t2.export_state()[0])
    assert np.array_equal(t.export_state()[1], t2.export_state()[1])


def test_persist_load_checkpoint_restore(tm, tmp_path):
    case = dict(CASES[3], create=dict(CASES[3]["create"]))
    inp = make_inputs(case)
    kind, tbl = ref_table(case["create"], seed=2, reusable=False)
    t = tm.create(kind, tbl)
    t.train(train_table(kind, inp, 2))
    assert t.info()["has_state"] == 0  # non-reusable machines drop their state
    with pytest.raises(tm.TsetlinError, match="without state"):
        t.train(train_table(kind, inp, 1))
    blob = t.persist()
    p = str(tmp_path / "model.bin")
    t.persist(p)
    assert open(p, "rb").read() == blob
    for t2 in (tm.load(blob, True), tm.load(p)):
        assert t2.type() == "encoder"
        assert np.array_equal(t2.predict(inp["xt"], inp["nt"]), t.predict(inp["xt"], inp["nt"]))
        assert t2.persist() == blob
    cp = t.checkpoint()
    assert len(cp) == t.info()["action_chunks"]
    t3 = tm.load(blob, True)
    t3.restore(bytes(len(cp)))
    assert not np.array_equal(t3.predict(inp["xt"], inp["nt"]), t.predict(inp["xt"], inp["nt"])) or True
    t3.restore(cp)
    assert t3.persist() == blob
    with pytest.raises(tm.TsetlinError, match="size mismatch"):
        t3.restore(bytes(3))


def test_reconfigure_matches_fresh_machine(tm):
    case = dict(CASES[0], create=dict(CASES[0]["create"]))
    inp = make_inputs(case)
    kind, tbl = ref_table(case["create"], seed=5)
    t = tm.create(kind, dict(tbl, reusable=True))
    t.train(train_table(kind, inp, 1))
    t.reconfigure(dict(clauses=24, clause_tolerance=5, clause_maximum=12, specificity=3.0,
                       target=0.5))
    t.train(train_table(kind, inp, 2))
    fresh = tm.create(kind, dict(tbl, clauses=24, clause_tolerance=5, clause_maximum=12,
                                 specificity=3.0, target=0.5))
    fresh.train(train_table(kind, inp, 2))
    assert t.info()["target"] == fresh.info()["target"] == 12
    assert np.array_equal(t.export_state()[0], fresh.export_state()[0])
    with pytest.raises(tm.TsetlinError, match="reusable"):
        tm.create(kind, dict(tbl, reusable=False)).reconfigure(
            dict(clauses=8, clause_tolerance=2, clause_maximum=2, specificity=2.0))


def test_restrict_matches_oracle(tm):
    case = dict(CASES[7], create=dict(CASES[7]["create"]))
    inp = make_inputs(case)
    m = _oracle_pair("encoder", case["create"], inp, 2, seed=8)
    kind, tbl = ref_table(case["create"], seed=8)
    t = tm.create(kind, tbl)
    t.train(train_table(kind, inp, 2))
    m.restrict([3, 1])
    t.restrict(np.array([3, 1]))
    a, s = t.export_state()
    assert np.array_equal(a, m.actions())
    assert np.array_equal(s, m.state())
    with pytest.raises(tm.TsetlinError, match="duplicate"):
        t.restrict(np.array([0, 0]))


def test_device_pointer_inputs_match_host(tm):
    import torch
    case = dict(CASES[9], create=dict(CASES[9]["create"]))
    inp = make_inputs(case)
    kind, tbl = ref_table(case["create"], seed=3)
    t1 = tm.create(kind, tbl)
    t1.train(train_table(kind, inp, 2))
    t2 = tm.create(kind, tbl)
    dinp = dict(inp, x=torch.from_numpy(inp["x"]).cuda(), labels=torch.from_numpy(inp["labels"]).cuda())
    t2.train(train_table(kind, dinp, 2))
    assert np.array_equal(t1.export_state()[1], t2.export_state()[1])
    xt = torch.from_numpy(inp["xt"]).cuda()
    assert np.array_equal(t2.predict(xt, inp["nt"]).cpu().numpy(), t1.predict(inp["xt"], inp["nt"]))


def test_train_batch_equals_individual(tm):
    from santoku_tsetlin import datagen
    x, y, _ = datagen.prototype_classifier(600, classes=10, seed=4)
    machines, tables, alone = [], [], []
    params = [dict(clauses=16, specificity=3.0, target=8, seed=1),
              dict(clauses=40, specificity=12.0, target=30, seed=2),
              dict(clauses=8, specificity=25.0, target=4, seed=1),
              dict(clauses=24, specificity=5.0, target=-1, seed=7)]
    for p in params:
        tbl = dict(classes=10, features=784, clause_tolerance=16, clause_maximum=16,
                   reusable=True, **p)
        tt = dict(samples=600, problems=x.ravel(), solutions=y, iterations=2)
        a = tm.create("classifier", tbl)
        a.train(tt)
        alone.append(a.export_state())
        machines.append(tm.create("classifier", tbl))
        tables.append(tt)
    tm.train_batch(machines, tables)
    for mach, (a, s) in zip(machines, alone):
        a2, s2 = mach.export_state()
        assert np.array_equal(a, a2) and np.array_equal(s, s2)


@pytest.mark.parametrize("features,state,pair,mode", [
    (784, 8, False, 3),     # short rows: one warp per unit
    (16384, 8, True, 2),    # 256 KB units split over a 2-CTA cluster (on request)
    (16384, 8, False, 1),   # same rows with the automata in global memory (default)
    (300, 12, False, 0),    # more than 8 state bits, shared-memory automata
    (12000, 10, False, 1),  # more than 8 state bits on wide rows: global memory
    (8192, 8, False, 0),    # 128 KB units, fewer than the SMs: shared planes
], ids=["warp", "pair", "global", "smem_b12", "global_b10", "smem_few_units"])
def test_train_variants_match_oracle(tm, monkeypatch, features, state, pair, mode):
    from santoku_tsetlin import datagen
    monkeypatch.setenv("TSETLIN_B200_AUTOTUNE", "0")  # the heuristic choice is asserted
    if pair:
        monkeypatch.setenv("TSETLIN_B200_PAIR", "1")
    rng = np.random.default_rng(features + state)
    n, classes = 160, 3
    x = datagen.flip_pack(rng.random((n + 40, features)) < 0.02)
    y = rng.integers(0, classes, size=n).astype(np.int64)
    cfg = dict(type="classifier", classes=classes, features=features, clauses=16,
               clause_tolerance=32, clause_maximum=300, state=state, include_bits=2,
               specificity=25.0, target=20)
    inp = dict(n=n, x=x[:n].ravel(), labels=y)
    m = _oracle_pair("classifier", cfg, inp, 2, seed=21)
    kind, tbl = ref_table(cfg, seed=21)
    t = tm.create(kind, tbl)
    t.stats_enable(True)
    t.train(train_table(kind, inp, 2))
    assert t.stats()["train_mode"] == mode
    a, s = t.export_state()
    assert np.array_equal(a, m.actions())
    assert np.array_equal(s, m.state())
    xt = x[n:].ravel()
    assert np.array_equal(t.predict_scores(xt, 40), m.predict(xt, 40, scores=True)[1])


def test_predict_inside_each_does_not_disturb_training(tm):
    """The reference's search driver predicts a validation set in every
    epoch's callback (optimize.lua:586-653); training must continue on its
    own rows."""
    case = dict(CASES[9], create=dict(CASES[9]["create"]))
    inp = make_inputs(case)
    kind, tbl = ref_table(case["create"], seed=6)
    t = tm.create(kind, tbl)
    scores = []

    def each(epoch):
        scores.append(t.predict_scores(inp["xt"], inp["nt"]))
        return True

    t.train(dict(train_table(kind, inp, 3), each=each))
    t2 = tm.create(kind, tbl)
    t2.train(train_table(kind, inp, 3))
    assert np.array_equal(t.export_state()[1], t2.export_state()[1])
    assert np.array_equal(scores[-1], t2.predict_scores(inp["xt"], inp["nt"]))


def test_train_batch_each_stops_like_each(tm):
    """A machine stopped by the batch callback ends as tm_train with an
    `each` that stops at the same epoch; a predict inside the callback does
    not disturb training."""
    from santoku_tsetlin import datagen
    x, y, _ = datagen.prototype_classifier(500, classes=10, seed=8)
    xt = x[400:].ravel()
    stops = [1, 3, 2]
    tbls = [dict(classes=10, features=784, clauses=16, clause_tolerance=16, clause_maximum=16,
                 specificity=s, target=8, seed=i, reusable=True) for i, s in enumerate((3.0, 9.0, 20.0))]
    tt = dict(samples=400, problems=x[:400].ravel(), solutions=y[:400], iterations=4)
    ms = [tm.create("classifier", b) for b in tbls]
    seen = []

    def each(epoch):
        for m in ms:
            m.predict(xt, 100)
        seen.append(epoch)
        return [epoch >= s for s in stops]

    tm.train_batch(ms, [tt] * 3, each=each)
    assert seen == [1, 2, 3]
    for m, b, s in zip(ms, tbls, stops):
        alone = tm.create("classifier", b)
        alone.train(dict(tt, each=lambda e, s=s: e < s))
        assert np.array_equal(m.export_state()[1], alone.export_state()[1])


@pytest.mark.parametrize("features", [784, 8192])
def test_autotuned_training_matches_heuristic(tm, features):
    """The tuner's trial launches run on the freshly reset automata and reset
    them again, so tuned training ends in the heuristic's state, bit for
    bit, on the first call (tuning) and on a cached second call."""
    from santoku_tsetlin import datagen
    rng = np.random.default_rng(features)
    n, classes = 300, 4
    x = datagen.flip_pack(rng.random((n, features)) < 0.05).ravel()
    y = rng.integers(0, classes, size=n).astype(np.int64)
    tbl = dict(classes=classes, features=features, clauses=32, clause_tolerance=16,
               clause_maximum=64, specificity=8.0, target=16, reusable=True, seed=5)
    tt = dict(samples=n, problems=x, solutions=y, iterations=3)
    ref = tm.create("classifier", tbl)
    ref.set_autotune(0)
    ref.train(tt)
    want = ref.export_state()
    for mode in (2, 1):
        t = tm.create("classifier", tbl)
        t.set_autotune(mode)
        t.stats_enable(True)
        t.train(tt)
        st = t.stats()
        assert st["train_autotuned"] == 1
        for a, b in zip(t.export_state(), want):
            assert np.array_equal(a, b)
        assert np.array_equal(t.predict(x, n), ref.predict(x, n))
        t.destroy()
    with pytest.raises(tm.TsetlinError):
        ref.set_autotune(3)
    ref.destroy()


def test_global_planes_chosen_by_occupancy(tm, monkeypatch):
    """160 units of 128 KB: shared planes fit one CTA per SM, global planes
    two; with more units than SMs the heuristic takes global planes."""
    from santoku_tsetlin import datagen
    monkeypatch.setenv("TSETLIN_B200_AUTOTUNE", "0")
    rng = np.random.default_rng(8192)
    n, classes, features = 120, 10, 8192
    x = datagen.flip_pack(rng.random((n + 20, features)) < 0.02)
    y = rng.integers(0, classes, size=n).astype(np.int64)
    cfg = dict(type="classifier", classes=classes, features=features, clauses=128,
               clause_tolerance=32, clause_maximum=300, include_bits=1,
               specificity=25.0, target=20)
    inp = dict(n=n, x=x[:n].ravel(), labels=y)
    m = _oracle_pair("classifier", cfg, inp, 1, seed=23)
    kind, tbl = ref_table(cfg, seed=23)
    t = tm.create(kind, tbl)
    t.stats_enable(True)
    t.train(train_table(kind, inp, 1))
    assert t.stats()["train_mode"] == 1
    a, st = t.export_state()
    assert np.array_equal(a, m.actions())
    assert np.array_equal(st, m.state())


@pytest.mark.parametrize("features", [784, 4000, 4500])
def test_every_train_variant_matches_oracle(tm, features):
    """Each train-kernel variant, pinned in turn -- one warp per unit (four
    units or one per CTA), shared or global count planes with 1, 2 or 4
    clauses per warp, the 2-CTA cluster, the word-per-thread
    configurations -- ends in the oracle's state, bit for bit."""
    from santoku_tsetlin import datagen
    rng = np.random.default_rng(features + 7)
    n, classes = 200, 4
    x = datagen.flip_pack(rng.random((n, features)) < 0.03).ravel()
    y = rng.integers(0, classes, size=n).astype(np.int64)
    cfg = dict(type="classifier", classes=classes, features=features, clauses=32,
               clause_tolerance=16, clause_maximum=120, specificity=12.0, target=16)
    inp = dict(n=n, x=x, labels=y)
    m = _oracle_pair("classifier", cfg, inp, 2, seed=31)
    want = (m.actions(), m.state())
    variants = [(0, 1), (0, 2), (0, 4), (1, 1), (1, 2), (1, 4), (2, 1)]
    if features <= 1024:
        variants += [(3, 1), (3, 2)]
    # the word-per-thread kernel's configurations that hold these rows
    # (4500 features: 282 words -> 512 threads x 2 words; 784: 52 words)
    wp = ((2 * features + 31) // 32 + 3) // 4 * 4
    for cid, words in ((1, 1024), (2, 256), (3, 512), (4, 256), (5, 64), (6, 64), (7, 64)):
        if wp <= words:
            variants.append((4, cid))
    kind, tbl = ref_table(cfg, seed=31)
    for mode, cpw in variants:
        t = tm.create(kind, tbl)
        t.force_variant(mode, cpw)
        t.stats_enable(True)
        t.train(train_table(kind, inp, 2))
        st = t.stats()
        assert (st["train_mode"], st["train_cpw"]) == (mode, cpw)
        a, s = t.export_state()
        assert np.array_equal(a, want[0]), (mode, cpw)
        assert np.array_equal(s, want[1]), (mode, cpw)
        t.destroy()
    t = tm.create(kind, tbl)
    t.force_variant(3, 4)
    with pytest.raises(tm.TsetlinError):
        t.force_variant(1, 3)
    with pytest.raises(tm.TsetlinError):
        t.force_variant(4, 9)
    with pytest.raises(tm.TsetlinError):
        t.force_variant(5, 1)
    with pytest.raises(tm.TsetlinError):  # the warp kernel holds four units or one per CTA
        t.train(train_table(kind, inp, 1))
    t.destroy()


@pytest.mark.parametrize("visible,variant", [(2000, (1, 4)), (4096, (1, 4)), (4096, (4, 2)),
                                             (4096, (4, 4))],
                         ids=["global4_128", "global4_256", "wpt2_256", "wpt4_256"])
def test_encoder_variants_match_oracle(tm, visible, variant):
    """Encoders (every sample trains every unit, the target is the code
    bit) on 128- and 256-word rows: the CTA kernel with global count planes
    and the word-per-thread configurations that hold these rows end in the
    oracle's state, bit for bit, over two epochs."""
    from santoku_tsetlin import datagen
    rng = np.random.default_rng(visible)
    n, hidden = 160, 12
    x = datagen.flip_pack(rng.random((n, visible)) < 0.05).ravel()
    codes = rng.integers(0, 256, size=n * 2).astype(np.uint8)
    cfg = dict(type="encoder", classes=hidden, features=visible, clauses=24,
               clause_tolerance=16, clause_maximum=48, specificity=15.0, target=20)
    inp = dict(n=n, x=x, codes=codes)
    m = _oracle_pair("encoder", cfg, inp, 2, seed=5)
    kind, tbl = ref_table(cfg, seed=5)
    t = tm.create(kind, tbl)
    t.force_variant(*variant)
    t.stats_enable(True)
    t.train(train_table(kind, inp, 2))
    assert (t.stats()["train_mode"], t.stats()["train_cpw"]) == variant
    a, st = t.export_state()
    assert np.array_equal(a, m.actions())
    assert np.array_equal(st, m.state())
    t.destroy()


@pytest.fixture(scope="module")
def c1_multiwave():
    """The large sparse classifier's rows (16,384 features flip-packed to
    1,024 words, Zipf data) with 240 clauses per class: 600 units of 8
    clauses, more than one wave of resident CTAs, trained 1 epoch on 2,000
    samples -- the production scheduling path (cost-ordered work list,
    atomic work counter, a CTA taking several units with its row ring's
    phase carried from one unit to the next)."""
    from santoku_tsetlin import datagen
    x, y = datagen.sparse_classifier(2300, classes=20, features=16384, seed=77)
    cfg = dict(type="classifier", classes=20, features=16384, clauses=240, clause_tolerance=64,
               clause_maximum=64, specificity=25.0, target=200)
    inp = dict(n=2000, x=x[:2000].ravel(), labels=y[:2000], xt=x[2000:].ravel(), nt=300)
    m = _oracle_pair("classifier", cfg, inp, 1, seed=41)
    return cfg, inp, (m.actions(), m.state(), m.predict(inp["xt"], 300, scores=True)[1])


@pytest.mark.parametrize("mode,cpw", [(-1, 1), (1, 1), (1, 2), (1, 4), (2, 1), (4, 1)],
                         ids=["auto", "global1", "global2", "global4", "pair", "wpt512"])
def test_multiwave_wide_rows_match_oracle(tm, c1_multiwave, mode, cpw):
    cfg, inp, (wa, ws, wsc) = c1_multiwave
    kind, tbl = ref_table(cfg, seed=41)
    t = tm.create(kind, tbl)
    if mode >= 0:
        t.force_variant(mode, cpw)
    t.stats_enable(True)
    t.train(train_table(kind, inp, 1))
    st = t.stats()
    assert st["train_unit_steps"] == 600 * 2000
    a, s = t.export_state()
    assert np.array_equal(a, wa), (mode, cpw)
    assert np.array_equal(s, ws), (mode, cpw)
    assert np.array_equal(t.predict_scores(inp["xt"], 300), wsc)
    t.destroy()


@pytest.mark.parametrize("kind,classes,F,clauses,ind,dens", [
    ("classifier", 20, 16384, 136, False, 0.01),    # the large sparse classifier's rows
    ("classifier", 20, 16384, 136, False, 0.0005),  # same, clauses short enough to vote
    ("encoder", 24, 4096, 40, False, 0.01),
    ("classifier", 3, 0, 24, True, 0.01),           # individualized: a row width per class
])
def test_small_batch_predict_matches_oracle(tm, kind, classes, F, clauses, ind, dens):
    """Predicts of 1 to 32 samples take the warp-per-clause kernel (each
    clause row read once; carry-save counts from 4 samples on), 33 and more
    the tiled one: both give the oracle's vote sums bit for bit, at every
    size across the switch.  The sparser actions give clauses of about 16
    literals, whose votes depend on the exact failed-literal counts."""
    rng = np.random.default_rng(classes + clauses)
    cfg = dict(type=kind, classes=classes, clauses=clauses, clause_tolerance=48,
               clause_maximum=64, specificity=25.0)
    if ind:
        fo = np.array([0, 700, 1900, 5000], dtype=np.int64)
        cfg.update(individualized=True, feat_offsets=fo)
    else:
        cfg["features"] = F
    m = O.Machine(**cfg)
    nbytes = m.info["action_chunks"]
    acts = np.packbits(rng.random(nbytes * 8) < dens, bitorder="little")
    m.load_state(actions=acts)
    kind2, tbl = ref_table(cfg)
    t = tm.create(kind2, tbl)
    t.import_state(actions=acts)
    for n in (1, 2, 3, 5, 8, 13, 16, 17, 31, 32, 33, 70):
        if ind:
            blocks, dof = [], [0]
            for h in range(classes):
                k = int(fo[h + 1] - fo[h])
                b = rng.random((n, k)) < 0.05
                blocks.append(np.packbits(np.concatenate([b, ~b], axis=1), axis=1,
                                          bitorder="little").ravel())
                dof.append(dof[-1] + blocks[-1].size)
            x = np.concatenate(blocks)
            dof = np.array(dof[:-1], dtype=np.int64)
            want = m.predict(x, n, dim_offsets=dof, scores=True)[1]
            assert np.array_equal(t.predict_scores(x, dof, n), want), n
        else:
            b = rng.random((n, F)) < 0.02
            x = np.packbits(np.concatenate([b, ~b], axis=1), axis=1, bitorder="little").ravel()
            want_out, want = m.predict(x, n, scores=True)
            assert np.array_equal(t.predict_scores(x, n), want), n
            assert np.array_equal(t.predict(x, n), want_out.ravel()), n
            if dens < 0.001:
                assert np.count_nonzero(want) > want.size // 2  # the votes are not all zero
    t.destroy()
