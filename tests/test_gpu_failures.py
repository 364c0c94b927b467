"""Failure paths, made on the host or by a wait that is told to give up --
no test here faults, traps or hangs the GPU.

* A sample-row wait that runs out: with TSETLIN_B200_ROW_WAIT=0 every
  thread of the fused train kernel gives up on its first row at once, the
  kernel sets its error status, drains the row copies it still has in
  flight (with the full wait limit) and returns; the train call reports
  TM_ERR_DEVICE and the context stays usable.
* Device allocations that fail (tm_debug_fail_alloc): create, train and
  predict report TM_ERR_OOM at every allocation they make, leak nothing
  that breaks the next call, and the machine trains bit-identically
  afterwards.
* A per-epoch callback that raises: the error is reported on stderr and
  training stops after that epoch, as the reference does with a Lua error
  in `each` (capi.c:1168-1182); the machine holds exactly the state of a
  training that ran that many epochs.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CFG = dict(classes=4, features=1100, clauses=16, clause_tolerance=16, clause_maximum=40,
           specificity=6.0, target=20, reusable=True, seed=3)


def _data(n=300, features=1100, classes=4, seed=4):
    from santoku_tsetlin import datagen
    x, y, _ = datagen.prototype_classifier(n, classes=classes, features=features, seed=seed)
    return x.ravel(), y.astype(np.int64)


@pytest.mark.parametrize("mode", [0, 1])
def test_row_wait_that_runs_out_reports_device_error(tm, mode, monkeypatch):
    x, y = _data()
    # rows of 1100 features are 69 words: the fused CTA-per-unit kernel with
    # TMA row copies (mode 0: automata in shared memory, 1: count planes in
    # global memory)
    monkeypatch.setenv("TSETLIN_B200_ROW_WAIT", "0")
    t = tm.create("classifier", dict(CFG))
    monkeypatch.delenv("TSETLIN_B200_ROW_WAIT")
    t.force_variant(mode, 1)
    with pytest.raises(tm.TsetlinError, match="did not complete"):
        t.train(dict(samples=len(y), problems=x, solutions=y, iterations=1))
    t.destroy()
    # the context is intact: a fresh machine trains and predicts normally,
    # and equals one trained by the other variant
    u = tm.create("classifier", dict(CFG))
    u.force_variant(mode, 1)
    u.train(dict(samples=len(y), problems=x, solutions=y, iterations=2))
    v = tm.create("classifier", dict(CFG))
    v.force_variant(1 - mode, 1)
    v.train(dict(samples=len(y), problems=x, solutions=y, iterations=2))
    ua, us = u.export_state()
    va, vs = v.export_state()
    assert np.array_equal(ua, va) and np.array_equal(us, vs)
    assert np.array_equal(u.predict(x, 50), v.predict(x, 50))


def _reference_state(tm, x, y, iterations=2):
    t = tm.create("classifier", dict(CFG))
    t.train(dict(samples=len(y), problems=x, solutions=y, iterations=iterations))
    a, s = t.export_state()
    p = t.predict(x, 40)
    t.destroy()
    return a, s, p


def test_allocation_failures_everywhere(tm):
    x, y = _data()
    want_a, want_s, want_p = _reference_state(tm, x, y)
    L = tm.lib()
    # create: fail each of its first allocations in turn
    seen_create = 0
    for k in range(12):
        L.tm_debug_fail_alloc(k)
        try:
            t = tm.create("classifier", dict(CFG))
        except tm.TsetlinError as e:
            assert "out of memory" in str(e) or "memory" in str(e).lower(), str(e)
            seen_create += 1
            continue
        finally:
            L.tm_debug_fail_alloc(-1)
        t.destroy()
    assert seen_create >= 3  # automata, count planes, class table, literal counts
    # train and predict: every allocation they make on a fresh machine, one
    # at a time
    seen_train = 0
    for k in range(16):
        t = tm.create("classifier", dict(CFG))
        L.tm_debug_fail_alloc(k)
        failed = False
        try:
            t.train(dict(samples=len(y), problems=x, solutions=y, iterations=2))
            t.predict(x, 40)
        except tm.TsetlinError as e:
            assert "memory" in str(e).lower(), str(e)
            failed = True
            seen_train += 1
        finally:
            L.tm_debug_fail_alloc(-1)
        # the same machine trains to the same state right after
        t.train(dict(samples=len(y), problems=x, solutions=y, iterations=2))
        a, s = t.export_state()
        assert np.array_equal(a, want_a) and np.array_equal(s, want_s), (k, failed)
        assert np.array_equal(t.predict(x, 40), want_p)
        t.destroy()
        if not failed:
            break
    assert seen_train >= 5  # rows, labels, class table, orders, sort, launch tables, ...


def test_raising_callback_stops_training_like_the_reference(tm, capfd):
    x, y = _data()
    t = tm.create("classifier", dict(CFG))
    seen = []

    def each(epoch):
        seen.append(epoch)
        if epoch == 2:
            raise RuntimeError("metric exploded")
        return True

    t.train(dict(samples=len(y), problems=x, solutions=y, iterations=5, each=each))
    assert seen == [1, 2]
    assert "metric exploded" in capfd.readouterr().err
    want_a, want_s, _ = _reference_state(tm, x, y, iterations=2)
    a, s = t.export_state()
    assert np.array_equal(a, want_a) and np.array_equal(s, want_s)
    # `false` stops the same way, without a message
    u = tm.create("classifier", dict(CFG))
    u.train(dict(samples=len(y), problems=x, solutions=y, iterations=5,
                 each=lambda e: e < 2))
    ua, us = u.export_state()
    assert np.array_equal(ua, want_a) and np.array_equal(us, want_s)


def test_raising_batch_callback_stops_every_machine(tm, capfd):
    x, y = _data()
    ms = [tm.create("classifier", dict(CFG, seed=s)) for s in (1, 2, 3)]
    tbl = dict(samples=len(y), problems=x, solutions=y, iterations=4)

    def each(epoch):
        if epoch == 1:
            raise ValueError("boom")
        return None

    tm.train_batch(ms, [dict(tbl) for _ in ms], each=each)
    assert "boom" in capfd.readouterr().err
    for m, s in zip(ms, (1, 2, 3)):
        r = tm.create("classifier", dict(CFG, seed=s))
        r.train(dict(tbl, iterations=1))
        assert np.array_equal(m.export_state()[1], r.export_state()[1])
