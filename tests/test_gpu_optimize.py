"""The search driver (optimize.lua restated): a batched round (all trials in
one train_batch with per-epoch control) gives exactly the per-trial scores,
epochs and chosen parameters of the sequential form; the final machine is
trained with the chosen parameters."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(tm):
    from santoku_tsetlin import datagen
    rs = np.random.default_rng(4242)
    base = rs.random(784) < 0.2
    protos = np.repeat(base[None], 10, axis=0)
    for c in range(10):
        protos[c, rs.choice(784, size=40, replace=False)] ^= True
    x, y, _ = datagen.prototype_classifier(1600, classes=10, features=784, flip=0.3, seed=5,
                                           prototypes=protos)
    xv, yv = x[1200:].ravel(), y[1200:]

    def metric(t):
        acc = tm.class_accuracy(t.predict(xv, len(yv)), yv, len(yv), 10)
        return acc["f1"], acc

    return dict(features=784, classes=10, samples=1200, problems=x[:1200].ravel(),
                solutions=y[:1200], search_metric=metric,
                holdout=dict(samples=len(yv), problems=xv, solutions=yv))


def test_batched_round_equals_sequential(tm):
    from santoku_tsetlin import optimize
    events = {True: [], False: []}
    results = {}
    for batched in (True, False):
        args = dict(_setup(tm), clauses={"def": 16, "min": 8, "max": 64, "round": 8},
                    clause_tolerance={"def": 16, "min": 8, "max": 64, "int": True},
                    clause_maximum={"def": 16, "min": 8, "max": 64, "int": True},
                    target={"def": 8, "min": 4, "max": 32, "int": True},
                    specificity={"def": 10, "min": 4, "max": 40},
                    include_bits=1, search_rounds=2, search_trials=4, search_iterations=4,
                    search_patience=2, final_iterations=3, final_patience=0, batched=batched,
                    search_seed=7,
                    each=lambda m, fin, met, p, e, r, t, b=batched: events[b].append(
                        (fin, r, t, e, round(met["f1"], 12))))
        final, metrics, best = optimize.classifier(args)
        results[batched] = (best, metrics["f1"])
        final.destroy()
    # per-trial epochs and scores: the batched callback interleaves trials
    # epoch by epoch, the sequential one runs them in order -- same multiset
    assert sorted(events[True]) == sorted(events[False])
    assert results[True] == results[False]
    assert any(e[0] for e in events[True])  # the final training ran


def test_device_metric_search_equals_callable(tm):
    """A search whose metric is a device metric table runs its batched
    rounds device-resident (train_batch_search) and chooses the same
    parameters, with the same final score, as the same search driven by the
    equivalent callable metric."""
    from santoku_tsetlin import optimize
    base = _setup(tm)
    results = {}
    for kind in ("callable", "device"):
        args = dict(base, clauses={"def": 16, "min": 8, "max": 64, "round": 8},
                    clause_tolerance={"def": 16, "min": 8, "max": 64, "int": True},
                    clause_maximum={"def": 16, "min": 8, "max": 64, "int": True},
                    target={"def": 8, "min": 4, "max": 32, "int": True},
                    specificity={"def": 10, "min": 4, "max": 40},
                    include_bits=1, search_rounds=2, search_trials=4, search_iterations=4,
                    search_patience=2, final_iterations=3, final_patience=0, batched=True,
                    search_seed=11)
        if kind == "device":
            args["search_metric"] = dict(base["holdout"], metric="f1")
        final, metrics, best = optimize.classifier(args)
        results[kind] = (best, metrics["f1"])
        final.destroy()
    assert results["device"] == results["callable"]
