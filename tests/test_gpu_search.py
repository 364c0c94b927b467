"""The device-resident search round (tm_train_batch_search) against the
reference's per-trial flow, run machine by machine on the host: train with
`each` = train_tm's epoch logic (optimize.lua:586-653, restated in
santoku_tsetlin.optimize._Tracker) and the search metric computed from
predict + the evaluator.  Per-epoch scores, stop epochs, final scores and
the final automata must be identical (scores are IEEE doubles computed in
the same order: the tolerance is zero)."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _params():
    # uneven machines: clauses, specificity, target, negated literals on/off
    return [dict(clauses=c, specificity=sp, target=tg, negated=ng, seed=i)
            for i, (c, sp, tg, ng) in enumerate([(16, 4.0, 20, True), (64, 12.0, 60, False),
                                                  (40, 25.0, 150, True), (8, 2.0, 30, False),
                                                  (128, 8.0, 100, True), (24, 30.0, 45, True)])]


@pytest.fixture(scope="module")
def data():
    from santoku_tsetlin import datagen
    protos = np.random.default_rng(5).random((10, 784)) < 0.2
    out = {}
    for neg in (True, False):
        x, y, _ = datagen.prototype_classifier(2300, classes=10, features=784, flip=0.3,
                                               seed=9, negated=neg, prototypes=protos)
        out[neg] = (x[:1500], y[:1500], x[1500:], y[1500:])
    return out


def _machine(tm, p):
    return tm.create("classifier", dict(classes=10, features=784 if p["negated"] else 392,
                                        clauses=p["clauses"], clause_tolerance=32,
                                        clause_maximum=64, specificity=p["specificity"],
                                        target=p["target"], seed=p["seed"], reusable=True))


def _sequential(tm, p, d, iters, patience, tolerance, metric):
    """The reference's flow for one trial: scores holds one score per
    epoch, then (after a restore) the restored machine's."""
    from santoku_tsetlin import optimize
    x, y, xv, yv = d[p["negated"]]
    m = _machine(tm, p)
    scores = []

    def metric_fn(t):
        pred = t.predict(xv.ravel(), len(yv))
        if metric == "f1":
            s = tm.class_accuracy(pred, yv, len(yv), 10)["f1"]
        else:
            s = float((pred == yv).sum()) / len(yv)
        scores.append(s)
        return s, None

    final, _ = optimize.train_tm("classifier", m, {"samples": len(y), "problems": x.ravel(),
                                                   "solutions": y},
                                 p, iters, patience, tolerance, metric_fn, None, {})
    return m, final, scores


def _epochs_of(scores, patience, tolerance, iters):
    best, since = -math.inf, 0
    for e, s in enumerate(scores):
        if s > best + tolerance:
            best, since = s, 0
        else:
            since += 1
        if (patience and since >= patience) or e + 1 >= iters:
            return e + 1
    return len(scores)


@pytest.mark.parametrize("metric,patience", [("f1", 2), ("accuracy", 1), ("f1", 0)])
def test_search_round_equals_sequential_train_tm(tm, data, metric, patience):
    iters, tol = 7, 1e-8
    ps = _params()
    ms = [_machine(tm, p) for p in ps]
    tables = [{"samples": 1500, "problems": data[p["negated"]][0].ravel(),
               "solutions": data[p["negated"]][1], "iterations": iters} for p in ps]
    # one round for all machines, each with the holdout of its literal layout
    r = tm.train_batch_search(ms, tables, {"samples": 800, "solutions": data[True][3],
                                           "problems_each": [data[p["negated"]][2].ravel()
                                                             for p in ps]},
                              patience=patience, tolerance=tol, metric=metric)
    for i, p in enumerate(ps):
        m, final, scores = _sequential(tm, p, data, iters, patience, tol, metric)
        n_ep = _epochs_of(scores, patience, tol, iters)
        assert int(r["epochs"][i]) == n_ep, (i, r["epochs"][i], n_ep)
        assert np.array_equal(r["scores"][i][:n_ep], np.array(scores[:n_ep])), i
        assert np.all(np.isnan(r["scores"][i][n_ep:]))
        assert r["final"][i] == final, (i, r["final"][i], final)
        a, s = ms[i].export_state()
        a2, s2 = m.export_state()
        assert np.array_equal(a, a2) and np.array_equal(s, s2), i
        m.destroy()
    for m in ms:
        m.destroy()


def test_search_round_encoder_mean_hamming(tm):
    from santoku_tsetlin import datagen, optimize
    x, c = datagen.latent_encoder(1300, visible=300, hidden=12, seed=4)
    xt, ct = x[1000:], c[1000:]
    cfgs = [dict(clauses=16, specificity=5.0, seed=1), dict(clauses=32, specificity=9.0, seed=2)]

    def make(cf):
        return tm.create("encoder", dict(hidden=12, visible=300, clauses=cf["clauses"],
                                         clause_tolerance=16, clause_maximum=40,
                                         specificity=cf["specificity"], seed=cf["seed"],
                                         reusable=True))
    ms = [make(cf) for cf in cfgs]
    tbl = {"samples": 1000, "sentences": x[:1000].ravel(), "codes": c[:1000].ravel(),
           "iterations": 5}
    r = tm.train_batch_search(ms, [dict(tbl) for _ in ms],
                              {"samples": 300, "sentences": xt.ravel(), "codes": ct.ravel()},
                              patience=2, metric="mean_hamming")
    for k, cf in enumerate(cfgs):
        m = make(cf)
        scores = []

        def metric_fn(t):
            s = tm.encoding_accuracy(t.predict(xt.ravel(), 300), ct.ravel(), 300, 12)
            scores.append(s["mean_hamming"])
            return s["mean_hamming"], None
        final, _ = optimize.train_tm("encoder", m, {"samples": 1000, "sentences": tbl["sentences"],
                                                    "codes": tbl["codes"]},
                                     cf, 5, 2, 1e-8, metric_fn, None, {})
        n_ep = int(r["epochs"][k])
        assert n_ep == _epochs_of(scores, 2, 1e-8, 5)
        assert np.array_equal(r["scores"][k][:n_ep], np.array(scores[:n_ep]))
        assert r["final"][k] == final
        a, s = ms[k].export_state()
        a2, s2 = m.export_state()
        assert np.array_equal(a, a2) and np.array_equal(s, s2)


def test_search_round_callback_stops_machines(tm, data):
    ps = [dict(p, negated=True) for p in _params()[:4]]
    ms = [_machine(tm, p) for p in ps]
    x, y, xv, yv = data[True]
    tbl = {"samples": 1500, "problems": x.ravel(), "solutions": y, "iterations": 6}
    seen = []

    def each(epoch, scores, training):
        seen.append((epoch, scores.copy(), training.copy()))
        return [epoch >= 2 and i % 2 == 0 for i in range(len(ms))]

    r = tm.train_batch_search(ms, [dict(tbl) for _ in ms],
                              {"samples": len(yv), "problems": xv.ravel(), "solutions": yv},
                              patience=0, each=each)
    assert list(r["epochs"]) == [2, 6, 2, 6]
    assert [e for e, _, _ in seen] == [1, 2, 3, 4, 5, 6]
    assert not np.isnan(seen[0][1]).any() and np.isnan(seen[2][1][0])
    for i, p in enumerate(ps):
        ref = _machine(tm, p)
        ref.train(dict(tbl, iterations=int(r["epochs"][i])))
        assert np.array_equal(ref.export_state()[1], ms[i].export_state()[1])


def test_search_round_device_inputs_and_stats(tm, data):
    import torch
    ps = [dict(p, negated=True) for p in _params()[:3]]
    ms = [_machine(tm, p) for p in ps]
    x, y, xv, yv = data[True]
    xd, yd = torch.from_numpy(x.ravel().copy()).cuda(), torch.from_numpy(y).cuda()
    xvd, yvd = torch.from_numpy(xv.ravel().copy()).cuda(), torch.from_numpy(yv).cuda()
    for m in ms:
        m.stats_enable(True)
    r = tm.train_batch_search(ms, [{"samples": 1500, "problems": xd, "solutions": yd,
                                    "iterations": 3} for _ in ms],
                              {"samples": len(yv), "problems": xvd, "solutions": yvd},
                              patience=0)
    h = tm.train_batch_search([_machine(tm, p) for p in ps],
                              [{"samples": 1500, "problems": x.ravel(), "solutions": y,
                                "iterations": 3} for _ in ms],
                              {"samples": len(yv), "problems": xv.ravel(), "solutions": yv},
                              patience=0)
    assert np.array_equal(r["scores"], h["scores"])
    st = ms[0].stats()
    assert st["search_epochs"] == 3 and st["search_epoch_ms"] > 0
    assert 0 < st["search_train_ms"] <= st["search_epoch_ms"]
    assert st["train_active_pairs"] > 0
